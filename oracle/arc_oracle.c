/*
 * arc_oracle.c - CPU restatement of arc-demo's batched world step.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker for the CUDA step in
 * arc_demo_b200/csrc; the product never links, loads or calls it. Only the
 * tests, the smoke check and bench.py's CPU-baseline leg use it.
 *
 * It restates, operation for operation, the reference's algorithm:
 *   csrc/arc_math.h      vector / quaternion helpers
 *   csrc/arc_rng.h       xorshift128 + hash seeding
 *   csrc/arc_terrain.c   block terrain generator and lookups
 *   csrc/arc_phys.c      substepped XPBD solver (arc_world_step)
 *   csrc/arc_robot.c     the quadruped template
 *   csrc/arc_sim.c       batched API: reset, step, observe, heights
 * Every floating-point expression keeps the reference's evaluation order, so
 * that the FP64 build, compiled without FMA contraction, is bitwise equal to
 * the reference compiled the same way (pinned by tests/test_oracle.py).
 *
 * Two builds come from this file:
 *   liboracle64.so  REAL = double: the reference's own arithmetic;
 *   liboracle32.so  REAL = float (-DORC_FP32): the physics step in FP32 with
 *                   the same operation order as the CUDA kernel. Set-up work
 *                   (robot template, terrain generation, reset poses, joint
 *                   limit sines/cosines) stays in FP64 and is rounded to FP32
 *                   once, exactly as the CUDA path does it.
 *
 * The only FP32-specific change of algorithm: the 3x3 solvers treat
 * |det| < 1e-30 (instead of 1e-300, which underflows in FP32) as singular.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef ORC_FP32
typedef float real;
#define R_SQRT sqrtf
#define R_ATAN2 atan2f
#define R_FABS fabsf
#define R_FLOOR floorf
#define R_TINY_DET 1e-30f
#define ORC_EXPORT(name) orc32_##name
#else
typedef double real;
#define R_SQRT sqrt
#define R_ATAN2 atan2
#define R_FABS fabs
#define R_FLOOR floor
#define R_TINY_DET 1e-300
#define ORC_EXPORT(name) orc64_##name
#endif

#define K(x) ((real)(x))
#define ORC_PI 3.14159265358979323846

/* capacities (csrc/arc_phys.h:19-23, csrc/arc_terrain.h:10) */
#define MAXB 16
#define MAXJ 16
#define MAXS 48
#define MAXC 128
#define GRID_MAX 64
#define NJ 12
#define NLEGS 4

/* ------------------------------------------------------------------------ */
/* FP64 helpers for set-up work (csrc/arc_math.h:20-137) */

typedef struct { double x, y, z; } d3;
typedef struct { double w, x, y, z; } dq;

static d3 d3v(double x, double y, double z) { d3 r; r.x = x; r.y = y; r.z = z; return r; }
static d3 d3_add(d3 a, d3 b) { return d3v(a.x + b.x, a.y + b.y, a.z + b.z); }
static d3 d3_sub(d3 a, d3 b) { return d3v(a.x - b.x, a.y - b.y, a.z - b.z); }
static d3 d3_scale(d3 a, double s) { return d3v(a.x * s, a.y * s, a.z * s); }
static d3 d3_madd(d3 a, d3 b, double s) { return d3v(a.x + b.x * s, a.y + b.y * s, a.z + b.z * s); }
static double d3_dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static d3 d3_cross(d3 a, d3 b)
{
    return d3v(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static double d3_len(d3 a) { return sqrt(d3_dot(a, a)); }
static d3 d3_normalize(d3 a)
{
    double l = d3_len(a);
    return l > 1e-15 ? d3_scale(a, 1.0 / l) : d3v(0.0, 0.0, 0.0);
}
static d3 d3_perp(d3 n) /* csrc/arc_math.h:61-65 */
{
    d3 t = fabs(n.x) < 0.57 ? d3v(1.0, 0.0, 0.0) : d3v(0.0, 1.0, 0.0);
    return d3_normalize(d3_cross(n, t));
}
static dq dqv(double w, double x, double y, double z) { dq r; r.w = w; r.x = x; r.y = y; r.z = z; return r; }
static dq dq_id(void) { return dqv(1.0, 0.0, 0.0, 0.0); }
static dq dq_conj(dq a) { return dqv(a.w, -a.x, -a.y, -a.z); }
static dq dq_mul(dq a, dq b)
{
    return dqv(a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z,
               a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
               a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
               a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w);
}
static dq dq_normalize(dq a)
{
    double l = sqrt(a.w * a.w + a.x * a.x + a.y * a.y + a.z * a.z);
    if (l < 1e-15)
        return dq_id();
    l = 1.0 / l;
    return dqv(a.w * l, a.x * l, a.y * l, a.z * l);
}
static dq dq_axis_angle(d3 axis, double angle)
{
    double s = sin(0.5 * angle);
    return dqv(cos(0.5 * angle), axis.x * s, axis.y * s, axis.z * s);
}
static d3 dq_rotate(dq q, d3 v)
{
    d3 u = d3v(q.x, q.y, q.z);
    d3 t = d3_scale(d3_cross(u, v), 2.0);
    return d3_add(d3_madd(v, t, q.w), d3_cross(u, t));
}
static d3 dq_inv_rotate(dq q, d3 v) { return dq_rotate(dq_conj(q), v); }

/* ------------------------------------------------------------------------ */
/* RNG (csrc/arc_rng.h:14-53): integer exact */

typedef struct { uint32_t s[4]; } orng;

static uint32_t rng_u32(orng *r)
{
    uint32_t t = r->s[3], s = r->s[0];
    r->s[3] = r->s[2];
    r->s[2] = r->s[1];
    r->s[1] = s;
    t = t ^ (t << 11);
    t ^= t >> 8;
    r->s[0] = t ^ s ^ (s >> 19);
    return r->s[0];
}

static uint32_t hash32(uint32_t x)
{
    x = (x ^ (x >> 16)) * 0x7feb352dU;
    x = (x ^ (x >> 15)) * 0x846ca68bU;
    return x ^ (x >> 16);
}

static void rng_seed(orng *r, uint32_t seed)
{
    int i;
    for (i = 0; i < 4; ++i) {
        seed = hash32(seed + 0x9e3779b9U * (uint32_t)(i + 1));
        r->s[i] = seed ? seed : 1U;
    }
}

static double rng_range(orng *r, double lo, double hi)
{
    return lo + (hi - lo) * (rng_u32(r) * (1.0 / 4294967296.0));
}

/* ------------------------------------------------------------------------ */
/* Terrain (csrc/arc_terrain.h:13-50, csrc/arc_terrain.c:17-71), in FP64 */

typedef struct {
    int nx, ny;
    double cell, ox, oy, outside;
    double h[GRID_MAX * GRID_MAX];
} dterrain;

static void terrain_flat(dterrain *t, int nx, int ny, double cell, double height)
{
    int i;
    if (nx > GRID_MAX) nx = GRID_MAX;
    if (ny > GRID_MAX) ny = GRID_MAX;
    t->nx = nx;
    t->ny = ny;
    t->cell = cell;
    t->ox = -0.5 * nx * cell;
    t->oy = -0.5 * ny * cell;
    t->outside = height;
    for (i = 0; i < nx * ny; ++i)
        t->h[i] = height;
}

static double dterrain_height(const dterrain *t, double x, double y)
{
    double fx = floor((x - t->ox) / t->cell), fy = floor((y - t->oy) / t->cell);
    if (!(fx >= 0.0 && fy >= 0.0 && fx < t->nx && fy < t->ny))
        return t->outside;
    return t->h[(int)fx + (int)fy * t->nx];
}

static double smooth(double t) { return t * t * (3.0 - 2.0 * t); }

static void add_noise(dterrain *t, int spacing, double amplitude, orng *rng)
{
    double lattice[(GRID_MAX / 3 + 3) * (GRID_MAX / 3 + 3)];
    int m = t->nx / spacing + 2, ix, iy;
    for (ix = 0; ix < m * m; ++ix)
        lattice[ix] = rng_range(rng, -1.0, 1.0);
    for (iy = 0; iy < t->ny; ++iy)
        for (ix = 0; ix < t->nx; ++ix) {
            double fx = (double)ix / spacing, fy = (double)iy / spacing;
            int gx = (int)fx, gy = (int)fy;
            double tx = smooth(fx - gx), ty = smooth(fy - gy);
            double a = lattice[gx + gy * m], b = lattice[gx + 1 + gy * m];
            double c = lattice[gx + (gy + 1) * m], d = lattice[gx + 1 + (gy + 1) * m];
            double v = (a + (b - a) * tx) * (1.0 - ty) + (c + (d - c) * tx) * ty;
            t->h[ix + iy * t->nx] += amplitude * v;
        }
}

static void terrain_generate(dterrain *t, int n, double cell, double difficulty, orng *rng)
{
    int i;
    double base;
    terrain_flat(t, n, n, cell, 0.0);
    t->outside = -100.0;
    if (difficulty <= 0.0)
        return;
    add_noise(t, 8, 0.45 * difficulty, rng);
    add_noise(t, 3, 0.12 * difficulty, rng);
    for (i = 0; i < t->nx * t->ny; ++i) {
        double h = t->h[i] + 0.06 * difficulty * rng_range(rng, -1.0, 1.0);
        t->h[i] = 0.03 * floor(h / 0.03 + 0.5);
    }
    base = dterrain_height(t, 0.0, 0.0);
    for (i = 0; i < t->nx * t->ny; ++i)
        t->h[i] -= base;
}

/* ------------------------------------------------------------------------ */
/* Robot template in FP64 (csrc/arc_robot.c:34-195, csrc/arc_phys.c:84-143) */

typedef struct {
    double mass, inv_mass;
    d3 inertia, inv_inertia;
    d3 x;
    dq q;
} tbody;

typedef struct {
    int parent, child;
    d3 r1, r2, a1, a2, b1, b2;
    dq q_rel0;
    double lo, hi, kp, kd, max_torque;
} tjoint;

typedef struct {
    int body;
    d3 pos;
    double radius;
} tsphere;

typedef struct {
    int nb, nj, ns;
    tbody b[MAXB];
    tjoint j[MAXJ];
    tsphere s[MAXS];
    d3 gravity;
    double mu_s, mu_d;
    /* robot info (csrc/arc_robot.h:22-30) */
    int foot_sphere[NLEGS], n_torso_spheres;
    double default_angles[NJ], lo[NJ], hi[NJ];
    double stand_height, total_mass, footprint;
} tmodel;

static int t_add_body(tmodel *m, double mass, d3 inertia, d3 pos, dq q)
{
    tbody *b;
    if (m->nb >= MAXB)
        return -1;
    b = &m->b[m->nb];
    memset(b, 0, sizeof(*b));
    b->x = pos;
    b->q = dq_normalize(q);
    b->mass = mass;
    b->inv_mass = 1.0 / mass;
    b->inertia = inertia;
    b->inv_inertia = d3v(1.0 / inertia.x, 1.0 / inertia.y, 1.0 / inertia.z);
    return m->nb++;
}

static int t_add_sphere(tmodel *m, int body, d3 pos, double radius)
{
    if (m->ns >= MAXS)
        return -1;
    m->s[m->ns].body = body;
    m->s[m->ns].pos = pos;
    m->s[m->ns].radius = radius;
    return m->ns++;
}

static int t_add_hinge(tmodel *m, int parent, int child, d3 anchor, d3 axis_world)
{
    tjoint *j;
    dq qp = dq_id(), qc;
    d3 xp = d3v(0.0, 0.0, 0.0), axis, ref;
    if (m->nj >= MAXJ || child <= parent)
        return -1;
    if (parent >= 0) {
        xp = m->b[parent].x;
        qp = m->b[parent].q;
    }
    qc = m->b[child].q;
    axis = d3_normalize(axis_world);
    ref = d3_perp(axis);
    j = &m->j[m->nj];
    memset(j, 0, sizeof(*j));
    j->parent = parent;
    j->child = child;
    j->r1 = dq_inv_rotate(qp, d3_sub(anchor, xp));
    j->r2 = dq_inv_rotate(qc, d3_sub(anchor, m->b[child].x));
    j->a1 = dq_inv_rotate(qp, axis);
    j->a2 = dq_inv_rotate(qc, axis);
    j->b1 = dq_inv_rotate(qp, ref);
    j->b2 = dq_inv_rotate(qc, ref);
    j->q_rel0 = dq_mul(dq_conj(qp), qc);
    j->lo = 1.0;
    j->hi = -1.0;
    return m->nj++;
}

/* Forward kinematics pose of every body (csrc/arc_phys.c:749-767); writes
 * body x, q into xs, qs. */
static void t_pose(const tmodel *m, d3 pos, dq q, const double *angles, d3 *xs, dq *qs)
{
    int i;
    xs[0] = pos;
    qs[0] = dq_normalize(q);
    for (i = 0; i < m->nj; ++i) {
        const tjoint *j = &m->j[i];
        d3 xp = j->parent >= 0 ? xs[j->parent] : d3v(0.0, 0.0, 0.0);
        dq qp = j->parent >= 0 ? qs[j->parent] : dq_id();
        d3 anchor = d3_add(xp, dq_rotate(qp, j->r1));
        qs[j->child] = dq_normalize(dq_mul(qp, dq_mul(dq_axis_angle(j->a1, angles[i]), j->q_rel0)));
        xs[j->child] = d3_sub(anchor, dq_rotate(qs[j->child], j->r2));
    }
}

static d3 inertia_sphere(double mass, double r)
{
    double i = 0.4 * mass * r * r;
    return d3v(i, i, i);
}

static d3 inertia_capsule_z(double mass, double radius, double half_length)
{
    double len = 2.0 * (half_length + radius);
    double ixx = mass * (3.0 * radius * radius + len * len) / 12.0;
    return d3v(ixx, ixx, 0.5 * mass * radius * radius);
}

static void set_drive(tjoint *j, double lo, double hi)
{
    j->lo = lo;
    j->hi = hi;
    j->kp = 250.0;
    j->kd = 6.0;
    j->max_torque = 80.0;
}

static void build_leg(tmodel *m, int leg, double sx, double sy)
{
    double psi = sx > 0.0 ? sy * 0.785 : sy * (ORC_PI - 0.785);
    d3 d = d3v(cos(psi), sin(psi), 0.0);
    d3 up = d3v(0.0, 0.0, 1.0);
    d3 lift = d3_cross(d, up);
    dq along = dq_axis_angle(d3_normalize(d3_cross(up, d)), 0.5 * ORC_PI);
    d3 hip = d3_add(d3_scale(d, 0.2 * cos(0.785)), d3v(0, 0, 0.2 * sin(0.785)));
    d3 p1 = d3_madd(hip, d, 0.06);
    d3 p2 = d3_madd(p1, d, 0.50);
    double fl = 0.5 * 0.50, tl = 0.5 * 0.95;
    int bc, bf, bt, j;
    bc = t_add_body(m, 0.4, d3v(0.02, 0.02, 0.02), d3_madd(hip, d, 0.5 * 0.06), dq_id());
    bf = t_add_body(m, 1.5, inertia_capsule_z(1.5, 0.06, fl), d3_madd(p1, d, fl), along);
    bt = t_add_body(m, 1.0, inertia_capsule_z(1.0, 0.05, tl), d3_madd(p2, d, tl), along);
    j = t_add_hinge(m, 0, bc, hip, d3v(0.0, 0.0, -sy));
    set_drive(&m->j[j], -0.8, 0.8);
    j = t_add_hinge(m, bc, bf, p1, lift);
    set_drive(&m->j[j], -0.4, 1.5);
    j = t_add_hinge(m, bf, bt, p2, lift);
    set_drive(&m->j[j], -2.8, -0.5);
    m->default_angles[3 * leg + 0] = 0.0;
    m->default_angles[3 * leg + 1] = 0.6;
    m->default_angles[3 * leg + 2] = -1.95;
    t_add_sphere(m, bf, d3v(0.0, 0.0, 0.0), 0.06);
    t_add_sphere(m, bt, d3v(0.0, 0.0, -tl), 0.07);
    t_add_sphere(m, bt, d3v(0.0, 0.0, -0.3 * tl), 0.055);
    t_add_sphere(m, bt, d3v(0.0, 0.0, 0.4 * tl), 0.035);
    m->foot_sphere[leg] = t_add_sphere(m, bt, d3v(0.0, 0.0, tl), 0.045);
}

static void build_robot(tmodel *m)
{
    static const double SX[NLEGS] = { 1.0, 1.0, -1.0, -1.0 };
    static const double SY[NLEGS] = { 1.0, -1.0, 1.0, -1.0 };
    d3 xs[MAXB];
    dq qs[MAXB];
    double lowest = 1e30;
    int leg, i;
    memset(m, 0, sizeof(*m));
    m->gravity = d3v(0.0, 0.0, -9.81);
    m->mu_s = 1.0;
    m->mu_d = 0.8;
    t_add_body(m, 8.0, inertia_sphere(8.0, 0.2), d3v(0, 0, 0), dq_id());
    t_add_sphere(m, 0, d3v(0, 0, 0), 0.2);
    m->n_torso_spheres = m->ns;
    for (leg = 0; leg < NLEGS; ++leg)
        build_leg(m, leg, SX[leg], SY[leg]);
    for (i = 0; i < NJ; ++i) {
        m->lo[i] = m->j[i].lo;
        m->hi[i] = m->j[i].hi;
    }
    m->total_mass = 0.0;
    for (i = 0; i < m->nb; ++i)
        m->total_mass += m->b[i].mass;
    t_pose(m, d3v(0, 0, 0), dq_id(), m->default_angles, xs, qs);
    m->footprint = 0.0;
    for (leg = 0; leg < NLEGS; ++leg) {
        const tsphere *s = &m->s[m->foot_sphere[leg]];
        d3 c = d3_add(xs[s->body], dq_rotate(qs[s->body], s->pos));
        lowest = lowest < c.z - s->radius ? lowest : c.z - s->radius;
        m->footprint += sqrt(c.x * c.x + c.y * c.y) / NLEGS;
    }
    m->stand_height = -lowest;
    t_pose(m, d3v(0, 0, m->stand_height), dq_id(), m->default_angles, xs, qs);
    for (i = 0; i < m->nb; ++i) {
        m->b[i].x = xs[i];
        m->b[i].q = qs[i];
    }
}

/* ------------------------------------------------------------------------ */
/* Step-precision vector math (csrc/arc_math.h:20-145) */

typedef struct { real x, y, z; } v3r;
typedef struct { real w, x, y, z; } qr;
typedef struct { real m[3][3]; } m3r;

static inline v3r v3(real x, real y, real z) { v3r r; r.x = x; r.y = y; r.z = z; return r; }
static inline v3r v_add(v3r a, v3r b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3r v_sub(v3r a, v3r b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3r v_scale(v3r a, real s) { return v3(a.x * s, a.y * s, a.z * s); }
static inline v3r v_neg(v3r a) { return v3(-a.x, -a.y, -a.z); }
static inline v3r v_mul(v3r a, v3r b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline v3r v_madd(v3r a, v3r b, real s) { return v3(a.x + b.x * s, a.y + b.y * s, a.z + b.z * s); }
static inline real v_dot(v3r a, v3r b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3r v_cross(v3r a, v3r b)
{
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline real v_len2(v3r a) { return v_dot(a, a); }
static inline real v_len(v3r a) { return R_SQRT(v_dot(a, a)); }
static inline qr qv(real w, real x, real y, real z) { qr r; r.w = w; r.x = x; r.y = y; r.z = z; return r; }
static inline qr q_conj(qr a) { return qv(a.w, -a.x, -a.y, -a.z); }
static inline qr q_mul(qr a, qr b)
{
    return qv(a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z,
              a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
              a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
              a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w);
}
static inline qr q_normalize(qr a)
{
    real l = R_SQRT(a.w * a.w + a.x * a.x + a.y * a.y + a.z * a.z);
    if (l < K(1e-15))
        return qv(K(1.0), K(0.0), K(0.0), K(0.0));
    l = K(1.0) / l;
    return qv(a.w * l, a.x * l, a.y * l, a.z * l);
}
static inline v3r q_rotate(qr q, v3r v)
{
    v3r u = v3(q.x, q.y, q.z);
    v3r t = v_scale(v_cross(u, v), K(2.0));
    return v_add(v_madd(v, t, q.w), v_cross(u, t));
}
static inline void m3_from_quat(m3r *r, qr q)
{
    real k = K(2.0) / (q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
    real x2 = q.x * k, y2 = q.y * k, z2 = q.z * k;
    real xx = q.x * x2, yy = q.y * y2, zz = q.z * z2;
    real xy = q.x * y2, xz = q.x * z2, yz = q.y * z2;
    real wx = q.w * x2, wy = q.w * y2, wz = q.w * z2;
    r->m[0][0] = K(1.0) - (yy + zz); r->m[0][1] = xy - wz;         r->m[0][2] = xz + wy;
    r->m[1][0] = xy + wz;         r->m[1][1] = K(1.0) - (xx + zz); r->m[1][2] = yz - wx;
    r->m[2][0] = xz - wy;         r->m[2][1] = yz + wx;         r->m[2][2] = K(1.0) - (xx + yy);
}
static inline v3r m3_mul_v3(const m3r *a, v3r v)
{
    return v3(a->m[0][0] * v.x + a->m[0][1] * v.y + a->m[0][2] * v.z,
              a->m[1][0] * v.x + a->m[1][1] * v.y + a->m[1][2] * v.z,
              a->m[2][0] * v.x + a->m[2][1] * v.y + a->m[2][2] * v.z);
}
static inline v3r m3_tmul_v3(const m3r *a, v3r v)
{
    return v3(a->m[0][0] * v.x + a->m[1][0] * v.y + a->m[2][0] * v.z,
              a->m[0][1] * v.x + a->m[1][1] * v.y + a->m[2][1] * v.z,
              a->m[0][2] * v.x + a->m[1][2] * v.y + a->m[2][2] * v.z);
}
static inline real r_min(real a, real b) { return a < b ? a : b; }
static inline real r_clamp(real v, real lo, real hi) { return v < lo ? lo : (v > hi ? hi : v); }

static v3r to_r3(d3 a) { return v3((real)a.x, (real)a.y, (real)a.z); }
static qr to_rq(dq a) { return qv((real)a.w, (real)a.x, (real)a.y, (real)a.z); }

/* ------------------------------------------------------------------------ */
/* World state (csrc/arc_phys.h:25-112), step precision */

typedef struct {
    v3r x, x_prev;
    qr q, q_prev;
    v3r v, w;
    real inv_mass;
    v3r inertia, inv_inertia;
    m3r rot, inv_iw;
} obody;

typedef struct {
    int parent, child;
    v3r r1, r2, a1, a2, b1, b2;
    real lo, hi, kp, kd, max_torque, target;
    real angle, rate, torque, torque_acc;
    real lim[4];
} ojoint;

typedef struct {
    int body;
    v3r pos;
    real radius;
    int touch, anchored;
    v3r anchor, anchor_n;
} osphere;

typedef struct {
    int body;
    v3r local, n;
} ocontact;

typedef struct {
    int nx, ny;
    real cell, ox, oy, outside;
    real h[GRID_MAX * GRID_MAX];
} oterrain;

typedef struct {
    v3r gravity;
    real mu_s, mu_d;
    int nb, nj, ns, nc, unstable;
    double time;
    obody b[MAXB];
    ojoint j[MAXJ];
    osphere s[MAXS];
    ocontact c[MAXC];
    oterrain t;
    /* Threshold margins of the last step. Test instrumentation: the tracing
     * only reads values the step computes and changes none of its
     * arithmetic. Per sphere, the closest call among its contact on/off
     * decisions (csrc/arc_phys.c:570, the buried-edge tests :572-581, :587),
     * in metres; per world, the closest friction-anchor reset (:519, the dot
     * product's distance from 0.9), static/dynamic friction (:534, relative
     * to the larger side) and joint-limit activation (:437-443, the sine
     * tests and the angle's distance from the bound, radians). */
    double m_contact[MAXS];
    double m_anchor, m_fric, m_limit;
} oworld;

/* margin tracing: m = min(m, |v|) */
static inline void tr_min(double *m, double v)
{
    v = fabs(v);
    if (v < *m)
        *m = v;
}

static inline int is_iso(v3r i) { return i.x == i.y && i.y == i.z; }

static inline real terrain_cell(const oterrain *t, int ix, int iy)
{
    if (ix < 0 || iy < 0 || ix >= t->nx || iy >= t->ny)
        return t->outside;
    return t->h[ix + iy * t->nx];
}

static inline real terrain_height(const oterrain *t, real x, real y)
{
    real fx = R_FLOOR((x - t->ox) / t->cell), fy = R_FLOOR((y - t->oy) / t->cell);
    if (!(fx >= K(0.0) && fy >= K(0.0) && fx < t->nx && fy < t->ny))
        return t->outside;
    return t->h[(int)fx + (int)fy * t->nx];
}

/* ------------------------------------------------------------------------ */
/* Solver (csrc/arc_phys.c:46-747) */

/* csrc/arc_phys.c:54-61 */
static inline qr q_turn(qr q, v3r w)
{
    real hx = K(0.5) * w.x, hy = K(0.5) * w.y, hz = K(0.5) * w.z;
    return qv(q.w - hx * q.x - hy * q.y - hz * q.z,
              q.x + hx * q.w + hy * q.z - hz * q.y,
              q.y - hx * q.z + hy * q.w + hz * q.x,
              q.z + hx * q.y - hy * q.x + hz * q.w);
}

/* csrc/arc_phys.c:64-82 */
static inline void body_sync(obody *b)
{
    v3r d = b->inv_inertia;
    int i, j;
    m3_from_quat(&b->rot, b->q);
    if (is_iso(d)) {
        memset(&b->inv_iw, 0, sizeof(b->inv_iw));
        b->inv_iw.m[0][0] = b->inv_iw.m[1][1] = b->inv_iw.m[2][2] = d.x;
        return;
    }
    for (i = 0; i < 3; ++i) {
        v3r rd = v3(b->rot.m[i][0] * d.x, b->rot.m[i][1] * d.y, b->rot.m[i][2] * d.z);
        for (j = i; j < 3; ++j)
            b->inv_iw.m[i][j] = b->inv_iw.m[j][i] =
                rd.x * b->rot.m[j][0] + rd.y * b->rot.m[j][1] + rd.z * b->rot.m[j][2];
    }
}

static inline v3r iiw(const obody *b, v3r v) { return m3_mul_v3(&b->inv_iw, v); }
static inline v3r brot(const obody *b, v3r v) { return b ? m3_mul_v3(&b->rot, v) : v; }

/* csrc/arc_phys.c:182-194 */
static inline real w_pos(const obody *b, v3r r, v3r n)
{
    v3r rn;
    if (!b)
        return K(0.0);
    rn = v_cross(r, n);
    return b->inv_mass + v_dot(rn, iiw(b, rn));
}
static inline real w_rot(const obody *b, v3r n) { return b ? v_dot(n, iiw(b, n)) : K(0.0); }

/* csrc/arc_phys.c:196-219 */
static inline void pos_impulse(obody *b, v3r r, v3r p)
{
    if (!b)
        return;
    b->x = v_madd(b->x, p, b->inv_mass);
    b->q = q_turn(b->q, iiw(b, v_cross(r, p)));
    body_sync(b);
}
static inline void rot_impulse(obody *b, v3r p)
{
    if (!b)
        return;
    b->q = q_turn(b->q, iiw(b, p));
    body_sync(b);
}
static inline void vel_impulse(obody *b, v3r r, v3r p)
{
    if (!b)
        return;
    b->v = v_madd(b->v, p, b->inv_mass);
    b->w = v_add(b->w, iiw(b, v_cross(r, p)));
}

/* csrc/arc_phys.c:226-242 */
static inline real solve_pos(obody *b1, v3r r1, obody *b2, v3r r2, v3r d, real alpha, real h)
{
    real c = v_len(d), denom, dl;
    v3r n, p;
    if (c < K(1e-12))
        return K(0.0);
    n = v_scale(d, K(1.0) / c);
    denom = w_pos(b1, r1, n) + w_pos(b2, r2, n) + alpha / (h * h);
    if (denom <= K(0.0))
        return K(0.0);
    dl = c / denom;
    p = v_scale(n, dl);
    pos_impulse(b1, r1, p);
    pos_impulse(b2, r2, v_neg(p));
    return dl;
}

/* csrc/arc_phys.c:245-262 */
static int solve3(const real Km[3][3], v3r d, v3r *x)
{
    real c00 = Km[1][1] * Km[2][2] - Km[1][2] * Km[2][1];
    real c01 = Km[1][2] * Km[2][0] - Km[1][0] * Km[2][2];
    real c02 = Km[1][0] * Km[2][1] - Km[1][1] * Km[2][0];
    real det = Km[0][0] * c00 + Km[0][1] * c01 + Km[0][2] * c02, inv;
    v3r c0, c1, c2;
    if (R_FABS(det) < R_TINY_DET)
        return 0;
    inv = K(1.0) / det;
    c0 = v3(Km[0][0], Km[1][0], Km[2][0]);
    c1 = v3(Km[0][1], Km[1][1], Km[2][1]);
    c2 = v3(Km[0][2], Km[1][2], Km[2][2]);
    x->x = v_dot(d, v_cross(c1, c2)) * inv;
    x->y = v_dot(c0, v_cross(d, c2)) * inv;
    x->z = v_dot(c0, v_cross(c1, d)) * inv;
    return 1;
}

/* csrc/arc_phys.c:265-280 */
static inline int solve3_sym(const real Km[3][3], v3r d, v3r *x)
{
    real a = Km[0][0], b = Km[0][1], c = Km[0][2], e = Km[1][1], f = Km[1][2], g = Km[2][2];
    real A = e * g - f * f, B = c * f - b * g, C = b * f - c * e;
    real det = a * A + b * B + c * C, inv, D, E, F;
    if (R_FABS(det) < R_TINY_DET)
        return 0;
    inv = K(1.0) / det;
    D = a * g - c * c;
    E = b * c - a * f;
    F = a * e - b * b;
    x->x = (A * d.x + B * d.y + C * d.z) * inv;
    x->y = (B * d.x + D * d.y + E * d.z) * inv;
    x->z = (C * d.x + E * d.y + F * d.z) * inv;
    return 1;
}

/* csrc/arc_phys.c:284-300 */
static inline void add_point_mass(real Km[3][3], const obody *b, v3r r)
{
    const m3r *a;
    real x = r.x, y = r.y, z = r.z, k01, k02, k12;
    if (!b)
        return;
    a = &b->inv_iw;
    Km[0][0] += b->inv_mass + a->m[1][1] * z * z - K(2.0) * a->m[1][2] * y * z + a->m[2][2] * y * y;
    Km[1][1] += b->inv_mass + a->m[2][2] * x * x - K(2.0) * a->m[0][2] * x * z + a->m[0][0] * z * z;
    Km[2][2] += b->inv_mass + a->m[0][0] * y * y - K(2.0) * a->m[0][1] * x * y + a->m[1][1] * x * x;
    k01 = a->m[1][2] * x * z + a->m[0][2] * y * z - a->m[0][1] * z * z - a->m[2][2] * x * y;
    k02 = a->m[0][1] * y * z + a->m[1][2] * x * y - a->m[1][1] * x * z - a->m[0][2] * y * y;
    k12 = a->m[0][2] * x * y + a->m[0][1] * x * z - a->m[0][0] * y * z - a->m[1][2] * x * x;
    Km[0][1] += k01; Km[1][0] += k01;
    Km[0][2] += k02; Km[2][0] += k02;
    Km[1][2] += k12; Km[2][1] += k12;
}

/* csrc/arc_phys.c:308-320 */
static inline void solve_point(obody *b1, v3r r1, obody *b2, v3r r2, v3r d)
{
    real Km[3][3] = { { 0, 0, 0 }, { 0, 0, 0 }, { 0, 0, 0 } };
    v3r p;
    if (v_len2(d) < K(1e-24))
        return;
    add_point_mass(Km, b1, r1);
    add_point_mass(Km, b2, r2);
    if (!solve3_sym((const real (*)[3])Km, d, &p))
        return;
    pos_impulse(b1, r1, p);
    pos_impulse(b2, r2, v_neg(p));
}

/* csrc/arc_phys.c:328-346 */
static inline void solve_rot_block(obody *b1, obody *b2, v3r rot)
{
    real Km[3][3] = { { 0, 0, 0 }, { 0, 0, 0 }, { 0, 0, 0 } };
    v3r p;
    int i, k;
    if (v_len2(rot) < K(1e-24))
        return;
    for (i = 0; i < 3; ++i)
        for (k = 0; k < 3; ++k) {
            if (b1)
                Km[i][k] += b1->inv_iw.m[i][k];
            if (b2)
                Km[i][k] += b2->inv_iw.m[i][k];
        }
    if (!solve3_sym((const real (*)[3])Km, rot, &p))
        return;
    rot_impulse(b1, p);
    rot_impulse(b2, v_neg(p));
}

/* csrc/arc_phys.c:353-371 */
static inline v3r solve_rot(obody *b1, obody *b2, v3r rot, real alpha, real h, real max_dl)
{
    real theta = v_len(rot), denom, dl;
    v3r n, p;
    if (theta < K(1e-12))
        return v3(0, 0, 0);
    n = v_scale(rot, K(1.0) / theta);
    denom = w_rot(b1, n) + w_rot(b2, n) + alpha / (h * h);
    if (denom <= K(0.0))
        return v3(0, 0, 0);
    dl = theta / denom;
    if (dl > max_dl)
        dl = max_dl;
    p = v_scale(n, dl);
    rot_impulse(b1, p);
    rot_impulse(b2, v_neg(p));
    return p;
}

static inline obody *jparent(oworld *w, const ojoint *j) { return j->parent >= 0 ? &w->b[j->parent] : 0; }
static inline qr body_q(const oworld *w, int i) { return i >= 0 ? w->b[i].q : qv(K(1.0), K(0.0), K(0.0), K(0.0)); }

/* csrc/arc_phys.c:386-400 */
static real joint_angle(const oworld *w, const ojoint *j)
{
    qr qp = body_q(w, j->parent), qc = body_q(w, j->child);
    v3r a = q_rotate(qp, j->a1);
    v3r b1 = q_rotate(qp, j->b1);
    v3r b2 = q_rotate(qc, j->b2);
    return R_ATAN2(v_dot(v_cross(b1, b2), a), v_dot(b1, b2));
}
static real joint_rate(const oworld *w, const ojoint *j)
{
    v3r a = q_rotate(body_q(w, j->parent), j->a1);
    v3r wp = j->parent >= 0 ? w->b[j->parent].w : v3(0, 0, 0);
    return v_dot(v_sub(w->b[j->child].w, wp), a);
}

/* csrc/arc_phys.c:404-411 */
static inline void joint_sincos(const obody *bp, const obody *bc, const ojoint *j, v3r a1, real *s, real *c)
{
    v3r b1 = brot(bp, j->b1);
    v3r b2 = brot(bc, j->b2);
    *s = v_dot(v_cross(b1, b2), a1);
    *c = v_dot(b1, b2);
}

/* csrc/arc_phys.c:413-457 */
static void joint_positions(oworld *w, ojoint *j, real h)
{
    obody *bp = jparent(w, j);
    obody *bc = &w->b[j->child];
    v3r a1, r1, r2, p1, p2;
    real phi, s, c;
    if (j->kp > K(0.0)) {
        v3r p;
        a1 = brot(bp, j->a1);
        joint_sincos(bp, bc, j, a1, &s, &c);
        phi = R_ATAN2(s, c);
        p = solve_rot(bp, bc, v_scale(a1, phi - j->target), K(1.0) / j->kp, h, j->max_torque * h * h);
        j->torque_acc -= v_dot(p, a1) / (h * h);
    }
    if (j->lo <= j->hi) {
        a1 = brot(bp, j->a1);
        joint_sincos(bp, bc, j, a1, &s, &c);
        tr_min(&w->m_limit, (double)(s * j->lim[0] - c * j->lim[1]));
        tr_min(&w->m_limit, (double)(j->lim[3] * c - j->lim[2] * s));
        if (j->hi - j->lo > K(ORC_PI) || s * j->lim[0] - c * j->lim[1] < K(0.0)
            || j->lim[3] * c - j->lim[2] * s < K(0.0)) {
            phi = R_ATAN2(s, c);
            tr_min(&w->m_limit, (double)(phi - j->lo));
            tr_min(&w->m_limit, (double)(phi - j->hi));
            if (phi < j->lo)
                solve_rot_block(bp, bc, v_scale(a1, phi - j->lo));
            else if (phi > j->hi)
                solve_rot_block(bp, bc, v_scale(a1, phi - j->hi));
        }
    }
    a1 = brot(bp, j->a1);
    solve_rot_block(bp, bc, v_cross(a1, brot(bc, j->a2)));
    r1 = brot(bp, j->r1);
    r2 = brot(bc, j->r2);
    p1 = bp ? v_add(bp->x, r1) : r1;
    p2 = v_add(bc->x, r2);
    solve_point(bp, r1, bc, r2, v_sub(p2, p1));
}

/* csrc/arc_phys.c:459-481 */
static void joint_velocities(oworld *w, ojoint *j, real h)
{
    obody *bp = jparent(w, j);
    obody *bc = &w->b[j->child];
    v3r a, wp;
    real rel, wsum, impulse, cap;
    if (j->kd <= K(0.0))
        return;
    a = brot(bp, j->a1);
    wp = bp ? bp->w : v3(0, 0, 0);
    rel = v_dot(v_sub(bc->w, wp), a);
    wsum = w_rot(bp, a) + w_rot(bc, a);
    if (wsum <= K(0.0))
        return;
    impulse = -j->kd * rel * h;
    cap = r_min(R_FABS(rel) / wsum, j->max_torque * h);
    impulse = r_clamp(impulse, -cap, cap);
    if (bp)
        bp->w = v_sub(bp->w, iiw(bp, v_scale(a, impulse)));
    bc->w = v_add(bc->w, iiw(bc, v_scale(a, impulse)));
    j->torque_acc += impulse / h;
}

/* csrc/arc_phys.c:488-500 */
static inline real solve_contact(oworld *w, int bi, v3r point, v3r n, real depth, real h)
{
    obody *b = &w->b[bi];
    v3r r = v_sub(point, b->x);
    real ln = solve_pos(b, r, 0, r, v_scale(n, depth), K(0.0), h);
    if (w->nc < MAXC) {
        ocontact *c = &w->c[w->nc++];
        c->body = bi;
        c->local = m3_tmul_v3(&b->rot, r);
        c->n = n;
    }
    return ln;
}

/* csrc/arc_phys.c:512-539 */
static inline void solve_friction(oworld *w, osphere *s, v3r n, real ln, real h)
{
    obody *b = &w->b[s->body];
    v3r c = v_add(b->x, brot(b, s->pos));
    v3r p = v_madd(c, n, -s->radius), e, r;
    real len, wt, lt, frac = K(1.0);
    if (s->anchored)
        tr_min(&w->m_anchor, (double)(v_dot(n, s->anchor_n) - K(0.9)));
    if (!s->anchored || v_dot(n, s->anchor_n) < K(0.9)) {
        v3r c0 = v_add(b->x_prev, q_rotate(b->q_prev, s->pos));
        s->anchor = v_madd(c0, n, -s->radius);
        s->anchor_n = n;
        s->anchored = 1;
    }
    e = v_sub(p, s->anchor);
    e = v_madd(e, n, -v_dot(e, n));
    len = v_len(e);
    if (len < K(1e-12))
        return;
    r = v_sub(p, b->x);
    wt = w_pos(b, r, v_scale(e, K(1.0) / len));
    lt = len / wt;
    {
        double a = fabs((double)lt), b = fabs((double)(w->mu_s * ln));
        tr_min(&w->m_fric, ((double)lt - (double)(w->mu_s * ln)) / (a > b ? (a > 1e-300 ? a : 1e-300) : b));
    }
    if (lt > w->mu_s * ln) {
        frac = r_min(w->mu_d * ln / lt, K(1.0));
        s->anchor = v_madd(s->anchor, e, K(1.0) - frac);
    }
    solve_pos(b, r, 0, r, v_scale(e, -frac), K(0.0), h);
}

/* csrc/arc_phys.c:542-610 */
static void collide_sphere(oworld *w, osphere *s, real h)
{
    const oterrain *t = &w->t;
    obody *b = &w->b[s->body];
    real rad = s->radius, ln = K(0.0);
    v3r c = v_add(b->x, brot(b, s->pos)), n_max = v3(0, 0, 1);
    real depth_max = K(0.0);
    int ix0, ix1, iy0, iy1, ix, iy, sx, sy, touched = 0;
    if (!(R_FABS(c.x) < K(1e6) && R_FABS(c.y) < K(1e6))) {
        s->anchored = 0;
        return;
    }
    ix0 = (int)R_FLOOR((c.x - rad - t->ox) / t->cell);
    ix1 = (int)R_FLOOR((c.x + rad - t->ox) / t->cell);
    iy0 = (int)R_FLOOR((c.y - rad - t->oy) / t->cell);
    iy1 = (int)R_FLOOR((c.y + rad - t->oy) / t->cell);
    for (iy = iy0; iy <= iy1; ++iy) {
        for (ix = ix0; ix <= ix1; ++ix) {
            real top = terrain_cell(t, ix, iy);
            real x0 = t->ox + ix * t->cell, x1 = x0 + t->cell;
            real y0 = t->oy + iy * t->cell, y1 = y0 + t->cell;
            real dist, depth;
            v3r q, diff, n;
            double *mc = &w->m_contact[s - w->s];
            tr_min(mc, (double)((c.z - rad) - top));
            if (c.z - rad >= top)
                continue;
            /* which neighbours the buried-edge tests read turns on c against
             * the column's edges wherever a neighbour on that side is at
             * least as high */
            if (terrain_cell(t, ix + 1, iy) >= top || terrain_cell(t, ix + 1, iy + 1) >= top ||
                terrain_cell(t, ix + 1, iy - 1) >= top)
                tr_min(mc, (double)(c.x - x1));
            if (terrain_cell(t, ix - 1, iy) >= top || terrain_cell(t, ix - 1, iy + 1) >= top ||
                terrain_cell(t, ix - 1, iy - 1) >= top)
                tr_min(mc, (double)(c.x - x0));
            if (terrain_cell(t, ix, iy + 1) >= top || terrain_cell(t, ix + 1, iy + 1) >= top ||
                terrain_cell(t, ix - 1, iy + 1) >= top)
                tr_min(mc, (double)(c.y - y1));
            if (terrain_cell(t, ix, iy - 1) >= top || terrain_cell(t, ix + 1, iy - 1) >= top ||
                terrain_cell(t, ix - 1, iy - 1) >= top)
                tr_min(mc, (double)(c.y - y0));
            sx = c.x > x1 ? 1 : (c.x < x0 ? -1 : 0);
            sy = c.y > y1 ? 1 : (c.y < y0 ? -1 : 0);
            if (sx && terrain_cell(t, ix + sx, iy) >= top)
                continue;
            if (sy && terrain_cell(t, ix, iy + sy) >= top)
                continue;
            if (sx && sy && terrain_cell(t, ix + sx, iy + sy) >= top)
                continue;
            q = v3(r_clamp(c.x, x0, x1), r_clamp(c.y, y0, y1), r_min(c.z, top));
            diff = v_sub(c, q);
            dist = v_len(diff);
            if (dist > K(1e-9)) {
                tr_min(mc, (double)(dist - rad));
                if (dist >= rad)
                    continue;
                n = v_scale(diff, K(1.0) / dist);
                depth = rad - dist;
            } else {
                n = v3(0, 0, 1);
                depth = top - c.z + rad;
            }
            ln += solve_contact(w, s->body, v_madd(c, n, -rad), n, depth, h);
            c = v_add(b->x, brot(b, s->pos));
            if (depth > depth_max) {
                depth_max = depth;
                n_max = n;
            }
            touched = 1;
        }
    }
    if (touched)
        solve_friction(w, s, n_max, ln, h);
    else
        s->anchored = 0;
    s->touch += touched;
}

/* csrc/arc_phys.c:612-626 */
static void contact_velocities(oworld *w)
{
    int i;
    for (i = 0; i < w->nc; ++i) {
        ocontact *c = &w->c[i];
        obody *b = &w->b[c->body];
        v3r r = brot(b, c->local);
        v3r vc = v_add(b->v, v_cross(b->w, r));
        real vn = v_dot(c->n, vc);
        vel_impulse(b, r, v_scale(c->n, -vn / w_pos(b, r, c->n)));
    }
}

/* csrc/arc_phys.c:636-656 */
static v3r gyroscopic(const obody *b, v3r w0, real h)
{
    real J[3][3];
    v3r iw = v_mul(w0, b->inertia), f = v_scale(v_cross(w0, iw), h), dw;
    real in[3];
    int k;
    in[0] = b->inertia.x;
    in[1] = b->inertia.y;
    in[2] = b->inertia.z;
    for (k = 0; k < 3; ++k) {
        v3r e = v3((real)(k == 0), (real)(k == 1), (real)(k == 2)), col;
        col = v_add(v_scale(e, in[k]),
                    v_scale(v_sub(v_scale(v_cross(w0, e), in[k]), v_cross(iw, e)), h));
        J[0][k] = col.x;
        J[1][k] = col.y;
        J[2][k] = col.z;
    }
    if (!solve3((const real (*)[3])J, f, &dw))
        return w0;
    return v_sub(w0, dw);
}

/* csrc/arc_phys.c:658-672 */
static void integrate(oworld *w, real h)
{
    int i;
    for (i = 0; i < w->nb; ++i) {
        obody *b = &w->b[i];
        b->x_prev = b->x;
        b->q_prev = b->q;
        b->v = v_madd(b->v, w->gravity, h);
        b->x = v_madd(b->x, b->v, h);
        if (!is_iso(b->inertia))
            b->w = m3_mul_v3(&b->rot, gyroscopic(b, m3_tmul_v3(&b->rot, b->w), h));
        b->q = q_turn(b->q, v_scale(b->w, h));
        body_sync(b);
    }
}

/* csrc/arc_phys.c:674-687 */
static void update_velocities(oworld *w, real h)
{
    int i;
    for (i = 0; i < w->nb; ++i) {
        obody *b = &w->b[i];
        qr dq;
        b->q = q_normalize(b->q);
        dq = q_mul(b->q, q_conj(b->q_prev));
        b->v = v_scale(v_sub(b->x, b->x_prev), K(1.0) / h);
        b->w = v_scale(v3(dq.x, dq.y, dq.z), K(2.0) / h);
        if (dq.w < K(0.0))
            b->w = v_neg(b->w);
    }
}

/* csrc/arc_phys.c:689-705 */
static int is_finite(real v) { return v == v && v < K(1e300) && v > K(-1e300); }

static void check_stability(oworld *w)
{
    int i;
    for (i = 0; i < w->nb; ++i) {
        obody *b = &w->b[i];
        real v2 = v_len2(b->v), w2 = v_len2(b->w);
        if (!is_finite(v2) || !is_finite(w2) || !(v_len2(b->x) < K(1e6) * K(1e6))
            || v2 > K(60.0) * K(60.0) || w2 > K(400.0) * K(400.0))
            w->unstable = 1;
    }
}

/* csrc/arc_phys.c:707-747. The joint limit sines and cosines are computed
 * in FP64 from the FP64 limits and rounded once (the CUDA path does the
 * same); for the FP64 build this is the reference's own computation. */
static void world_step(oworld *w, const double (*lim64)[4], double dt, int substeps)
{
    real h = (real)(dt / substeps);
    int s, i;
    for (i = 0; i < w->nb; ++i)
        body_sync(&w->b[i]);
    for (i = 0; i < w->ns; ++i) {
        w->s[i].touch = 0;
        w->m_contact[i] = 1e30;
    }
    w->m_anchor = w->m_fric = w->m_limit = 1e30;
    for (i = 0; i < w->nj; ++i) {
        ojoint *j = &w->j[i];
        j->torque_acc = K(0.0);
        j->lim[0] = (real)lim64[i][0];
        j->lim[1] = (real)lim64[i][1];
        j->lim[2] = (real)lim64[i][2];
        j->lim[3] = (real)lim64[i][3];
    }
    for (s = 0; s < substeps; ++s) {
        integrate(w, h);
        w->nc = 0;
        for (i = 0; i < w->nj; ++i)
            joint_positions(w, &w->j[i], h);
        for (i = 0; i < w->ns; ++i)
            collide_sphere(w, &w->s[i], h);
        update_velocities(w, h);
        for (i = 0; i < w->nj; ++i)
            joint_velocities(w, &w->j[i], h);
        contact_velocities(w);
    }
    for (i = 0; i < w->nj; ++i) {
        ojoint *j = &w->j[i];
        j->angle = joint_angle(w, j);
        j->rate = joint_rate(w, j);
        j->torque = j->torque_acc / (real)substeps;
    }
    w->time += dt;
    check_stability(w);
}

/* ------------------------------------------------------------------------ */
/* Batched simulation (csrc/arc_sim.c:11-215) */

typedef struct {
    int n, substeps, grid;
    double dt, cell;
    tmodel model;
    double lim64[MAXJ][4];
    int channel[MAXS];
    oworld tmpl;
    oworld *worlds;
    double (*geom64)[4];  /* per world: cell, ox, oy, outside in FP64 */
} osim;

/* Copies the FP64 model (bodies as built, flat terrain) into a step world. */
static void world_from_model(oworld *w, const tmodel *m)
{
    int i;
    memset(w, 0, sizeof(*w));
    w->gravity = to_r3(m->gravity);
    w->mu_s = (real)m->mu_s;
    w->mu_d = (real)m->mu_d;
    w->nb = m->nb;
    w->nj = m->nj;
    w->ns = m->ns;
    for (i = 0; i < m->nb; ++i) {
        obody *b = &w->b[i];
        b->x = b->x_prev = to_r3(m->b[i].x);
        b->q = b->q_prev = to_rq(m->b[i].q);
        b->inv_mass = (real)m->b[i].inv_mass;
        b->inertia = to_r3(m->b[i].inertia);
        b->inv_inertia = to_r3(m->b[i].inv_inertia);
        body_sync(b);
    }
    for (i = 0; i < m->nj; ++i) {
        ojoint *j = &w->j[i];
        const tjoint *t = &m->j[i];
        j->parent = t->parent;
        j->child = t->child;
        j->r1 = to_r3(t->r1); j->r2 = to_r3(t->r2);
        j->a1 = to_r3(t->a1); j->a2 = to_r3(t->a2);
        j->b1 = to_r3(t->b1); j->b2 = to_r3(t->b2);
        j->lo = (real)t->lo; j->hi = (real)t->hi;
        j->kp = (real)t->kp; j->kd = (real)t->kd;
        j->max_torque = (real)t->max_torque;
    }
    for (i = 0; i < m->ns; ++i) {
        osphere *s = &w->s[i];
        s->body = m->s[i].body;
        s->pos = to_r3(m->s[i].pos);
        s->radius = (real)m->s[i].radius;
    }
}

static void load_terrain(oterrain *t, const dterrain *d)
{
    int i;
    t->nx = d->nx;
    t->ny = d->ny;
    t->cell = (real)d->cell;
    t->ox = (real)d->ox;
    t->oy = (real)d->oy;
    t->outside = (real)d->outside;
    for (i = 0; i < d->nx * d->ny; ++i)
        t->h[i] = (real)d->h[i];
}

/* csrc/arc_sim.c:88-110: seeded terrain, noisy stance, random yaw, drop
 * height from the footprint; all in FP64, rounded into the world. */
static void reset_world(const osim *s, oworld *w, double *geom, uint32_t seed, double difficulty)
{
    const tmodel *m = &s->model;
    orng rng;
    dterrain t;
    double angles[NJ], ground = -1e30, yaw, x, y, reach;
    d3 xs[MAXB];
    dq qs[MAXB];
    int i;
    rng_seed(&rng, seed);
    terrain_generate(&t, s->grid, s->cell, difficulty, &rng);
    for (i = 0; i < NJ; ++i) {
        double a = m->default_angles[i] + rng_range(&rng, -0.1, 0.1);
        angles[i] = a < m->lo[i] ? m->lo[i] : (a > m->hi[i] ? m->hi[i] : a);
    }
    yaw = rng_range(&rng, -ORC_PI, ORC_PI);
    reach = m->footprint + 0.1;
    for (x = -reach; x <= reach; x += 0.5 * s->cell)
        for (y = -reach; y <= reach; y += 0.5 * s->cell) {
            double g = dterrain_height(&t, x, y);
            ground = ground > g ? ground : g;
        }
    t_pose(m, d3v(0.0, 0.0, ground + m->stand_height + 0.03),
           dq_axis_angle(d3v(0.0, 0.0, 1.0), yaw), angles, xs, qs);
    /* template copy (everything but the terrain), then the pose */
    memcpy(w, &s->tmpl, offsetof(oworld, t));
    load_terrain(&w->t, &t);
    geom[0] = t.cell;
    geom[1] = t.ox;
    geom[2] = t.oy;
    geom[3] = t.outside;
    for (i = 0; i < m->nb; ++i) {
        obody *b = &w->b[i];
        b->x = b->x_prev = to_r3(xs[i]);
        b->q = b->q_prev = to_rq(qs[i]);
        b->v = v3(0, 0, 0);
        b->w = v3(0, 0, 0);
        body_sync(b);
    }
    for (i = 0; i < m->nj; ++i) {
        ojoint *j = &w->j[i];
        j->target = j->angle = (real)angles[i];
        j->rate = j->torque = K(0.0);
    }
    for (i = 0; i < m->ns; ++i) {
        w->s[i].touch = 0;
        w->s[i].anchored = 0;
    }
    w->nc = 0;
    w->unstable = 0;
}

#define EXPORT __attribute__((visibility("default")))

EXPORT osim *ORC_EXPORT(create)(int n, double dt, int substeps, int grid, double cell)
{
    osim *s = (osim *)calloc(1, sizeof(osim));
    dterrain flat;
    int i;
    if (!s)
        return 0;
    s->n = n;
    s->dt = dt;
    s->substeps = substeps;
    s->grid = grid < GRID_MAX ? grid : GRID_MAX;
    s->cell = cell;
    s->worlds = (oworld *)malloc(sizeof(oworld) * (size_t)(n > 0 ? n : 1));
    s->geom64 = (double (*)[4])malloc(sizeof(double[4]) * (size_t)(n > 0 ? n : 1));
    if (!s->worlds || !s->geom64) {
        free(s->worlds);
        free(s->geom64);
        free(s);
        return 0;
    }
    build_robot(&s->model);
    for (i = 0; i < s->model.nj; ++i) {
        s->lim64[i][0] = cos(s->model.j[i].lo);
        s->lim64[i][1] = sin(s->model.j[i].lo);
        s->lim64[i][2] = cos(s->model.j[i].hi);
        s->lim64[i][3] = sin(s->model.j[i].hi);
    }
    for (i = 0; i < s->model.ns; ++i)
        s->channel[i] = i < s->model.n_torso_spheres ? NLEGS : NLEGS + 1;
    for (i = 0; i < NLEGS; ++i)
        s->channel[s->model.foot_sphere[i]] = i;
    world_from_model(&s->tmpl, &s->model);
    /* the template's pose sets the drive targets (csrc/arc_robot.c:194) */
    for (i = 0; i < s->model.nj; ++i)
        s->tmpl.j[i].target = s->tmpl.j[i].angle = (real)s->model.default_angles[i];
    terrain_flat(&flat, s->grid, s->grid, cell, 0.0);
    load_terrain(&s->tmpl.t, &flat);
    for (i = 0; i < n; ++i) {
        memcpy(&s->worlds[i], &s->tmpl, sizeof(oworld));
        s->geom64[i][0] = flat.cell;
        s->geom64[i][1] = flat.ox;
        s->geom64[i][2] = flat.oy;
        s->geom64[i][3] = flat.outside;
    }
    return s;
}

EXPORT void ORC_EXPORT(destroy)(osim *s)
{
    if (!s)
        return;
    free(s->worlds);
    free(s->geom64);
    free(s);
}

EXPORT int ORC_EXPORT(num_worlds)(const osim *s) { return s->n; }
EXPORT int ORC_EXPORT(real_size)(void) { return (int)sizeof(real); }

EXPORT void ORC_EXPORT(robot_info)(const osim *s, double *def, double *lo, double *hi, double *misc)
{
    int i;
    for (i = 0; i < NJ; ++i) {
        if (def) def[i] = s->model.default_angles[i];
        if (lo) lo[i] = s->model.lo[i];
        if (hi) hi[i] = s->model.hi[i];
    }
    if (misc) {
        misc[0] = s->model.stand_height;
        misc[1] = s->model.total_mass;
        misc[2] = s->model.footprint;
    }
}

EXPORT void ORC_EXPORT(reset)(osim *s, const int *ids, int n_ids, const unsigned *seeds,
                              const double *difficulty)
{
    int k;
#pragma omp parallel for schedule(static)
    for (k = 0; k < n_ids; ++k)
        reset_world(s, &s->worlds[ids[k]], s->geom64[ids[k]], seeds[k], difficulty[k]);
}

EXPORT void ORC_EXPORT(step)(osim *s, const double *targets)
{
    int i;
#pragma omp parallel for schedule(static)
    for (i = 0; i < s->n; ++i) {
        oworld *w = &s->worlds[i];
        int j;
        for (j = 0; j < NJ; ++j)
            w->j[j].target = r_clamp((real)targets[i * NJ + j], w->j[j].lo, w->j[j].hi);
        if (!w->unstable)
            world_step(w, (const double (*)[4])s->lim64, s->dt, s->substeps);
    }
}

/* Steps only the listed worlds (the rest keep their state). */
EXPORT void ORC_EXPORT(step_some)(osim *s, const int *ids, int n_ids, const double *targets)
{
    int k;
#pragma omp parallel for schedule(static)
    for (k = 0; k < n_ids; ++k) {
        int i = ids[k], j;
        oworld *w = &s->worlds[i];
        for (j = 0; j < NJ; ++j)
            w->j[j].target = r_clamp((real)targets[i * NJ + j], w->j[j].lo, w->j[j].hi);
        if (!w->unstable)
            world_step(w, (const double (*)[4])s->lim64, s->dt, s->substeps);
    }
}

/* csrc/arc_sim.c:140-183 */
EXPORT void ORC_EXPORT(observe)(const osim *s, double *root, double *rot, double *joints,
                                double *contacts, int *flags)
{
    int i;
#pragma omp parallel for schedule(static)
    for (i = 0; i < s->n; ++i) {
        const oworld *w = &s->worlds[i];
        const obody *b = &w->b[0];
        int j;
        if (root) {
            double *r = root + (size_t)i * 13;
            r[0] = b->x.x; r[1] = b->x.y; r[2] = b->x.z;
            r[3] = b->q.w; r[4] = b->q.x; r[5] = b->q.y; r[6] = b->q.z;
            r[7] = b->v.x; r[8] = b->v.y; r[9] = b->v.z;
            r[10] = b->w.x; r[11] = b->w.y; r[12] = b->w.z;
        }
        if (rot) {
            /* FP64 from the state, as the reference's read-out (csrc/arc_sim.c:158-162) */
            double qw = b->q.w, qx = b->q.x, qy = b->q.y, qz = b->q.z;
            double k = 2.0 / (qw * qw + qx * qx + qy * qy + qz * qz);
            double x2 = qx * k, y2 = qy * k, z2 = qz * k;
            double xx = qx * x2, yy = qy * y2, zz = qz * z2;
            double xy = qx * y2, xz = qx * z2, yz = qy * z2;
            double wx = qw * x2, wy = qw * y2, wz = qw * z2;
            double *o = rot + (size_t)i * 9;
            o[0] = 1.0 - (yy + zz); o[1] = xy - wz;         o[2] = xz + wy;
            o[3] = xy + wz;         o[4] = 1.0 - (xx + zz); o[5] = yz - wx;
            o[6] = xz - wy;         o[7] = yz + wx;         o[8] = 1.0 - (xx + yy);
        }
        if (joints) {
            double *o = joints + (size_t)i * 3 * NJ;
            for (j = 0; j < NJ; ++j) {
                o[j] = w->j[j].angle;
                o[NJ + j] = w->j[j].rate;
                o[2 * NJ + j] = w->j[j].torque;
            }
        }
        if (contacts) {
            double *o = contacts + (size_t)i * (NLEGS + 2), inv = 1.0 / s->substeps;
            for (j = 0; j < NLEGS + 2; ++j)
                o[j] = 0.0;
            for (j = 0; j < w->ns; ++j) {
                double *c = &o[s->channel[j]], v = w->s[j].touch * inv;
                *c = *c > v ? *c : v;
            }
        }
        if (flags)
            flags[i] = w->unstable;
    }
}

/* Height of the column under (x, y) in FP64 (csrc/arc_terrain.h:42-50),
 * over the step-precision heights. */
static double height64(const oterrain *t, const double *geom, double x, double y)
{
    double fx = floor((x - geom[1]) / geom[0]), fy = floor((y - geom[2]) / geom[0]);
    if (!(fx >= 0.0 && fy >= 0.0 && fx < t->nx && fy < t->ny))
        return geom[3];
    return t->h[(int)fx + (int)fy * t->nx];
}

/* csrc/arc_sim.c:185-203, in FP64 from the step-precision state (the
 * reference's read-out arithmetic; the CUDA path does the same). */
EXPORT void ORC_EXPORT(heights)(const osim *s, const double *offsets, int k, double *out)
{
    int i;
#pragma omp parallel for schedule(static)
    for (i = 0; i < s->n; ++i) {
        const oworld *w = &s->worlds[i];
        const obody *b = &w->b[0];
        d3 fwd = dq_rotate(dqv(b->q.w, b->q.x, b->q.y, b->q.z), d3v(1.0, 0.0, 0.0));
        double yaw = atan2(fwd.y, fwd.x), c = cos(yaw), sn = sin(yaw);
        double px = b->x.x, py = b->x.y;
        int j;
        for (j = 0; j < k; ++j) {
            double f = offsets[2 * j], l = offsets[2 * j + 1];
            out[(size_t)i * k + j] = height64(&w->t, s->geom64[i], px + c * f - sn * l, py + sn * f + c * l);
        }
    }
}

/* csrc/arc_sim.c:205-210 */
EXPORT void ORC_EXPORT(terrain_at)(const osim *s, const int *ids, const double *xy, int m, double *out)
{
    int i;
    for (i = 0; i < m; ++i)
        out[i] = height64(&s->worlds[ids[i]].t, s->geom64[ids[i]], xy[2 * i], xy[2 * i + 1]);
}

/* ------------------------------------------------------------------------ */
/* State snapshots for teacher forcing and fixtures. One world's dynamic
 * state as 387 doubles: bodies (x3 q4 v3 w3) x13, spheres (anchored,
 * anchor3, anchor_n3, touch) x21, joints (target, angle, rate, torque) x12,
 * unstable, time. The CUDA library uses the same layout. */

#define SNAP_BODY 13
#define SNAP_SPHERE 8
#define SNAP_JOINT 4

EXPORT int ORC_EXPORT(state_size)(const osim *s)
{
    return s->model.nb * SNAP_BODY + s->model.ns * SNAP_SPHERE + s->model.nj * SNAP_JOINT + 2;
}

/* Threshold margins of each world's last step (see oworld): per world, ns
 * contact margins, then the anchor, friction and limit margins (1e30: no
 * such decision was taken). */
EXPORT void ORC_EXPORT(margins)(const osim *s, double *out)
{
    int i, k;
    for (i = 0; i < s->n; ++i) {
        const oworld *w = &s->worlds[i];
        double *o = out + (size_t)i * (w->ns + 3);
        for (k = 0; k < w->ns; ++k)
            o[k] = w->m_contact[k];
        o[w->ns] = w->m_anchor;
        o[w->ns + 1] = w->m_fric;
        o[w->ns + 2] = w->m_limit;
    }
}

EXPORT void ORC_EXPORT(get_state)(const osim *s, const int *ids, int n_ids, double *out)
{
    int k, stride = ORC_EXPORT(state_size)(s);
    for (k = 0; k < n_ids; ++k) {
        const oworld *w = &s->worlds[ids[k]];
        double *o = out + (size_t)k * stride;
        int i;
        for (i = 0; i < w->nb; ++i) {
            const obody *b = &w->b[i];
            *o++ = b->x.x; *o++ = b->x.y; *o++ = b->x.z;
            *o++ = b->q.w; *o++ = b->q.x; *o++ = b->q.y; *o++ = b->q.z;
            *o++ = b->v.x; *o++ = b->v.y; *o++ = b->v.z;
            *o++ = b->w.x; *o++ = b->w.y; *o++ = b->w.z;
        }
        for (i = 0; i < w->ns; ++i) {
            const osphere *sp = &w->s[i];
            *o++ = sp->anchored;
            *o++ = sp->anchor.x; *o++ = sp->anchor.y; *o++ = sp->anchor.z;
            *o++ = sp->anchor_n.x; *o++ = sp->anchor_n.y; *o++ = sp->anchor_n.z;
            *o++ = sp->touch;
        }
        for (i = 0; i < w->nj; ++i) {
            const ojoint *j = &w->j[i];
            *o++ = j->target; *o++ = j->angle; *o++ = j->rate; *o++ = j->torque;
        }
        *o++ = w->unstable;
        *o++ = w->time;
    }
}

EXPORT void ORC_EXPORT(set_state)(osim *s, const int *ids, int n_ids, const double *in)
{
    int k, stride = ORC_EXPORT(state_size)(s);
    for (k = 0; k < n_ids; ++k) {
        oworld *w = &s->worlds[ids[k]];
        const double *p = in + (size_t)k * stride;
        int i;
        for (i = 0; i < w->nb; ++i) {
            obody *b = &w->b[i];
            b->x = v3((real)p[0], (real)p[1], (real)p[2]);
            b->q = qv((real)p[3], (real)p[4], (real)p[5], (real)p[6]);
            b->v = v3((real)p[7], (real)p[8], (real)p[9]);
            b->w = v3((real)p[10], (real)p[11], (real)p[12]);
            b->x_prev = b->x;
            b->q_prev = b->q;
            p += SNAP_BODY;
        }
        for (i = 0; i < w->ns; ++i) {
            osphere *sp = &w->s[i];
            sp->anchored = p[0] != 0.0;
            sp->anchor = v3((real)p[1], (real)p[2], (real)p[3]);
            sp->anchor_n = v3((real)p[4], (real)p[5], (real)p[6]);
            sp->touch = (int)p[7];
            p += SNAP_SPHERE;
        }
        for (i = 0; i < w->nj; ++i) {
            ojoint *j = &w->j[i];
            j->target = (real)p[0]; j->angle = (real)p[1]; j->rate = (real)p[2]; j->torque = (real)p[3];
            p += SNAP_JOINT;
        }
        w->unstable = p[0] != 0.0;
        w->time = p[1];
    }
}

/* Terrain of one world: grid size, cell, heights (nx*ny, row-major in y);
 * the grid is centred on the origin and surrounded by `outside`. */
EXPORT void ORC_EXPORT(set_terrain)(osim *s, int id, int nx, int ny, double cell, double outside,
                                    const double *heights)
{
    dterrain t;
    int i;
    terrain_flat(&t, nx, ny, cell, 0.0);
    t.outside = outside;
    for (i = 0; i < t.nx * t.ny; ++i)
        t.h[i] = heights[i];
    load_terrain(&s->worlds[id].t, &t);
    s->geom64[id][0] = t.cell;
    s->geom64[id][1] = t.ox;
    s->geom64[id][2] = t.oy;
    s->geom64[id][3] = t.outside;
}

EXPORT void ORC_EXPORT(get_terrain)(const osim *s, int id, int *nxy, double *geom, double *heights)
{
    const oterrain *t = &s->worlds[id].t;
    int i;
    nxy[0] = t->nx;
    nxy[1] = t->ny;
    for (i = 0; i < 4; ++i)
        geom[i] = s->geom64[id][i];
    if (heights)
        for (i = 0; i < t->nx * t->ny; ++i)
            heights[i] = t->h[i];
}

/* Terrain generator alone, for golden checks: n x n heights. */
EXPORT void ORC_EXPORT(terrain_generate)(int n, double cell, double difficulty, unsigned seed,
                                         double *out, double *geom)
{
    dterrain t;
    orng rng;
    int i;
    rng_seed(&rng, seed);
    terrain_generate(&t, n, cell, difficulty, &rng);
    for (i = 0; i < t.nx * t.ny; ++i)
        out[i] = t.h[i];
    if (geom) {
        geom[0] = t.nx;
        geom[1] = t.cell;
        geom[2] = t.ox;
        geom[3] = t.outside;
    }
}

/* The template constants, for checks of the CUDA library's copy:
 * per body (mass, inertia3, x3, q4) = 11, per joint (parent, child, r1, r2,
 * a1, a2, b1, b2, q_rel0, lo, hi, kp, kd, max_torque) = 29, per sphere
 * (body, pos3, radius) = 5. Returns the number of doubles written. */
EXPORT int ORC_EXPORT(model_dump)(const osim *s, double *out)
{
    const tmodel *m = &s->model;
    double *o = out;
    int i;
    for (i = 0; i < m->nb; ++i) {
        const tbody *b = &m->b[i];
        *o++ = b->mass;
        *o++ = b->inertia.x; *o++ = b->inertia.y; *o++ = b->inertia.z;
        *o++ = b->x.x; *o++ = b->x.y; *o++ = b->x.z;
        *o++ = b->q.w; *o++ = b->q.x; *o++ = b->q.y; *o++ = b->q.z;
    }
    for (i = 0; i < m->nj; ++i) {
        const tjoint *j = &m->j[i];
        const d3 *v[6];
        int k;
        v[0] = &j->r1; v[1] = &j->r2; v[2] = &j->a1; v[3] = &j->a2; v[4] = &j->b1; v[5] = &j->b2;
        *o++ = j->parent;
        *o++ = j->child;
        for (k = 0; k < 6; ++k) {
            *o++ = v[k]->x; *o++ = v[k]->y; *o++ = v[k]->z;
        }
        *o++ = j->q_rel0.w; *o++ = j->q_rel0.x; *o++ = j->q_rel0.y; *o++ = j->q_rel0.z;
        *o++ = j->lo; *o++ = j->hi; *o++ = j->kp; *o++ = j->kd; *o++ = j->max_torque;
    }
    for (i = 0; i < m->ns; ++i) {
        const tsphere *sp = &m->s[i];
        *o++ = sp->body;
        *o++ = sp->pos.x; *o++ = sp->pos.y; *o++ = sp->pos.z;
        *o++ = sp->radius;
    }
    return (int)(o - out);
}

/* Number of contacts recorded in the last substep of world i. */
EXPORT int ORC_EXPORT(n_contacts)(const osim *s, int i) { return s->worlds[i].nc; }
