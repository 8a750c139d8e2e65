/*
 * render_oracle.c - CPU restatement of arc-demo's renderer, for checking
 * the GPU ray caster (arc_demo_b200/csrc/arc_render.cu).
 *
 * TEST INFRASTRUCTURE ONLY. The product never links, loads or calls this
 * file; only the tests and bench.py's CPU-baseline leg use it.
 *
 * Parity is unpinned against the reference itself: its renderer
 * (csrc/arc_render.c, csrc/arc_mesh.c) needs SDL2 and OpenGL 2.1, which
 * cannot run on these machines. This file restates the same scene in double
 * precision from those sources, with the ray-casting model the GPU renderer
 * documents (exact or sphere-traced shapes instead of meshes, a shadow ray
 * instead of the shadow map, the 4x multisample pattern shaded once per
 * pixel and surface, ray-differential derivatives), written independently of the
 * CUDA code and by brute force:
 *   - every terrain column is a box from the void's bottom to its top,
 *     tested against every ray (the GPU walks a 2D DDA over the cells);
 *   - every visual is tested against every ray (the GPU culls them per tile);
 *   - the rounded box and torus are sphere traced to 1e-7 m in double.
 * Only the shader's hash of lattice points and the dither are evaluated in
 * float with the GPU's operation order, because sin() of arguments near
 * 5e4 times 43758 amplifies any rounding difference into a different value.
 *
 * Sources followed: csrc/arc_render.c:93-263 (look and fragment shader),
 * :280-302 (glow shader), :313-319 (vignette), :523-549 (lamps),
 * :566-672 (markers, glow billboards), :700-716 (camera), :962-968 (views),
 * :986-1062 (shadow square, lights, projection); csrc/arc_mesh.c (shapes,
 * terrain colours and ambient occlusion).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "arc_world.h"

#define PI 3.14159265358979323846

typedef struct { double x, y, z; } v3;

static v3 V(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static v3 add(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 sub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 mul(v3 a, double s) { return V(a.x * s, a.y * s, a.z * s); }
static v3 hadamard(v3 a, v3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
static double dot3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static v3 crs(v3 a, v3 b) { return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static double norm(v3 a) { return sqrt(dot3(a, a)); }
static v3 unit(v3 a) { double l = norm(a); return l > 1e-15 ? mul(a, 1.0 / l) : V(0, 0, 0); }
static double clampd(double x, double lo, double hi) { return x < lo ? lo : (x > hi ? hi : x); }
static double lerp(double a, double b, double t) { return a + (b - a) * t; }
static double sstep(double e0, double e1, double x)
{
    double t = clampd((x - e0) / (e1 - e0), 0.0, 1.0);
    return t * t * (3.0 - 2.0 * t);
}
static double fract_d(double x) { return x - floor(x); }

/* rotation matrix of a unit quaternion, world = R local */
static void quat_mat(arcw_quat q, double m[9])
{
    m[0] = 1 - 2 * (q.y * q.y + q.z * q.z);
    m[1] = 2 * (q.x * q.y - q.w * q.z);
    m[2] = 2 * (q.x * q.z + q.w * q.y);
    m[3] = 2 * (q.x * q.y + q.w * q.z);
    m[4] = 1 - 2 * (q.x * q.x + q.z * q.z);
    m[5] = 2 * (q.y * q.z - q.w * q.x);
    m[6] = 2 * (q.x * q.z - q.w * q.y);
    m[7] = 2 * (q.y * q.z + q.w * q.x);
    m[8] = 1 - 2 * (q.x * q.x + q.y * q.y);
}
static v3 mv(const double m[9], v3 a)
{
    return V(m[0] * a.x + m[1] * a.y + m[2] * a.z, m[3] * a.x + m[4] * a.y + m[5] * a.z,
             m[6] * a.x + m[7] * a.y + m[8] * a.z);
}
static v3 mtv(const double m[9], v3 a)
{
    return V(m[0] * a.x + m[3] * a.y + m[6] * a.z, m[1] * a.x + m[4] * a.y + m[7] * a.z,
             m[2] * a.x + m[5] * a.y + m[8] * a.z);
}
static v3 cv(arcw_vec3 a) { return V(a.x, a.y, a.z); }

/* ---- the shader's float hash, with the GPU's rounding order */
static float hash_f(float x, float y)
{
    float s = sinf(fmaf(x, 127.1f, y * 311.7f)) * 43758.5453f;
    return s - floorf(s);
}
static double vnoise(double x, double y)
{
    double ix = floor(x), iy = floor(y), fx = x - ix, fy = y - iy;
    fx = fx * fx * (3.0 - 2.0 * fx);
    fy = fy * fy * (3.0 - 2.0 * fy);
    double a = lerp(hash_f((float)ix, (float)iy), hash_f((float)ix + 1.0f, (float)iy), fx);
    double b = lerp(hash_f((float)ix, (float)iy + 1.0f), hash_f((float)ix + 1.0f, (float)iy + 1.0f), fx);
    return lerp(a, b, fy);
}

/* ---- scene */

enum { SPHERE, BOX, TAPER, CYLINDER, RING };
enum { M_PAINT, M_PANELS, M_METAL, M_RUBBER, M_LENS, M_RIBS, M_GLOW };
static const double MAT[7][4] = {{0.45, 36, 0, 0}, {0.50, 40, 0, 2}, {0.90, 64, 0, 0}, {0.08, 10, 0, 0},
                                 {1.80, 180, 0, 0}, {0.60, 40, 0, 0}, {0.00, 1, 3, 0}};
static const double SUN_C[3] = {1.45, 1.55, 1.80}, FILL_C[3] = {0.16, 0.13, 0.11}, LAMP_C[3] = {0.40, 0.30, 0.20};
static const double SKY[3] = {0.090, 0.100, 0.125}, GND[3] = {0.030, 0.030, 0.034};
static const float SEEN_F[3] = {1.00f, 0.42f, 0.08f}, UNSEEN_F[3] = {0.20f, 0.55f, 1.00f};

typedef struct {       /* a shape in world space */
    int type, material, robot, glow;
    double col[3];
    double m[9];       /* body rotation (world = m local + x) */
    v3 x;
    /* body-frame geometry */
    v3 p0, p1, axis, u, w;
    double r, r2, aspect, len, bevel;
    v3 inner;
    v3 pn[10];
    double pw[10];
} shape;

typedef struct {
    int nx, ny;
    double cell, ox, oy, outside, lo, hi, bottom;
    const double *h;
    v3 eye, fwd, right, up, target;
    double tan_y, aspect, fog_start, focus[2];
    float time_frac;
    v3 sun, fill, sl, ul;
    double sc[2];
    v3 lamps[9];
    v3 eye_pos, eye_dir, eye_col, beacon_pos, beacon_col;
    int ns;
    shape s[80 + 8];
    int ng;
    struct { v3 c, col, side; double s, alpha; int beam; } g[32];
} scene;

static double cell_at(const scene *S, int ix, int iy)
{
    if (ix < 0 || iy < 0 || ix >= S->nx || iy >= S->ny)
        return S->outside;
    return S->h[ix + iy * S->nx];
}

static double height_at(const scene *S, double x, double y)
{
    double fx = floor((x - S->ox) / S->cell), fy = floor((y - S->oy) / S->cell);
    if (!(fx >= 0.0 && fy >= 0.0 && fx < S->nx && fy < S->ny))
        return S->outside;
    return S->h[(int)fx + (int)fy * S->nx];
}

static void frame_of_segment(v3 p0, v3 p1, v3 *d, v3 *u, v3 *w, double *L)
{
    v3 s = sub(p1, p0);
    *L = norm(s);
    *d = mul(s, 1.0 / (*L > 1e-12 ? *L : 1.0));
    if (fabs(d->x) < 1e-9 && fabs(d->y) < 1e-9) {
        *u = V(1, 0, 0);
        *w = V(0, d->z > 0 ? 1 : -1, 0);
    } else {
        *u = unit(fabs(d->z) < 0.9 ? crs(V(0, 0, 1), *d) : crs(V(1, 0, 0), *d));
        *w = crs(*d, *u);
    }
}

/* body-frame shape from a visual; returns 0 for a degenerate one */
static int shape_of(const arcw_visual *v, shape *s)
{
    static const double PX[8] = {1, 0.6, -0.6, -1, -1, -0.6, 0.6, 1};
    static const double PY[8] = {0.45, 1, 1, 0.45, -0.45, -1, -1, -0.45};
    s->type = v->type;
    s->material = v->material;
    s->glow = v->material == M_GLOW;
    s->p0 = cv(v->p0);
    s->p1 = cv(v->p1);
    s->r = v->radius;
    s->r2 = v->radius2;
    s->aspect = v->aspect;
    for (int k = 0; k < 3; ++k)
        s->col[k] = v->color[k];
    if (v->type == BOX) {
        double e = fmin(v->p1.x, fmin(v->p1.y, v->p1.z));
        s->bevel = 0.22 * e;
        s->inner = V(v->p1.x - s->bevel, v->p1.y - s->bevel, v->p1.z - s->bevel);
    } else if (v->type == TAPER || v->type == CYLINDER) {
        frame_of_segment(s->p0, s->p1, &s->axis, &s->u, &s->w, &s->len);
        if (s->len < 1e-9)
            return 0;
        if (v->type == TAPER) {
            v3 a[8], b[8];
            for (int k = 0; k < 8; ++k) {
                a[k] = add(s->p0, add(mul(s->u, PX[k] * s->r), mul(s->w, PY[k] * s->r * s->aspect)));
                b[k] = add(add(s->p0, mul(s->axis, s->len)),
                           add(mul(s->u, PX[k] * s->r2), mul(s->w, PY[k] * s->r2 * s->aspect)));
            }
            for (int k = 0; k < 8; ++k) {
                v3 n = unit(crs(sub(a[(k + 1) % 8], a[k]), sub(b[k], a[k])));
                if (dot3(n, sub(a[k], s->p0)) < 0.0)
                    n = mul(n, -1.0);
                s->pn[k] = n;
                s->pw[k] = dot3(n, a[k]);
            }
            s->pn[8] = mul(s->axis, -1.0);
            s->pw[8] = -dot3(s->axis, s->p0);
            s->pn[9] = s->axis;
            s->pw[9] = dot3(s->axis, add(s->p0, mul(s->axis, s->len)));
        }
    } else if (v->type == RING) {
        s->axis = unit(s->p1);
    } else if (v->type != SPHERE) {
        return 0;
    }
    return 1;
}

/* ---- intersections in the body frame; unit direction d; nearest t in (1e-4, tmax) */

static double sdf_rbox(const shape *s, v3 q)
{
    double ax = fabs(q.x) - s->inner.x, ay = fabs(q.y) - s->inner.y, az = fabs(q.z) - s->inner.z;
    double ox = fmax(ax, 0), oy = fmax(ay, 0), oz = fmax(az, 0);
    return sqrt(ox * ox + oy * oy + oz * oz) + fmin(fmax(ax, fmax(ay, az)), 0.0) - s->bevel;
}

static double sdf_torus(const shape *s, v3 w)
{
    double h = dot3(w, s->axis);
    double rho = norm(sub(w, mul(s->axis, h))) - s->r;
    return sqrt(rho * rho + h * h) - s->r2;
}

static int march(const shape *s, v3 o, v3 d, double t0, double t1, double *t, int torus)
{
    double tt = t0;
    for (int i = 0; i < 400; ++i) {
        v3 q = add(sub(o, s->p0), mul(d, tt));
        double dist = torus ? sdf_torus(s, q) : sdf_rbox(s, q);
        if (dist < 1e-7) {
            *t = tt;
            return 1;
        }
        tt += dist;
        if (tt > t1)
            return 0;
    }
    return 0;
}

static int sphere_hit(v3 c, double r, v3 o, v3 d, double tmax, double *t)
{
    v3 oc = sub(o, c);
    double b = dot3(oc, d), disc = b * b - (dot3(oc, oc) - r * r);
    if (disc < 0)
        return 0;
    double q = sqrt(disc), ta = -b - q;
    if (ta <= 1e-4)
        ta = -b + q;
    if (ta <= 1e-4 || ta >= tmax)
        return 0;
    *t = ta;
    return 1;
}

/* body-frame hit: t, body-frame normal */
static int shape_hit(const shape *s, v3 o, v3 d, double tmax, double *t, v3 *n)
{
    switch (s->type) {
    case SPHERE:
        if (!sphere_hit(s->p0, s->r, o, d, tmax, t))
            return 0;
        *n = unit(sub(add(o, mul(d, *t)), s->p0));
        return 1;
    case BOX: {
        double r = norm(V(s->inner.x + s->bevel, s->inner.y + s->bevel, s->inner.z + s->bevel));
        v3 oc = sub(o, s->p0);
        double b = dot3(oc, d), disc = b * b - (dot3(oc, oc) - r * r);
        if (disc < 0)
            return 0;
        double t0 = fmax(-b - sqrt(disc), 1e-4), t1 = fmin(-b + sqrt(disc), tmax);
        if (t0 > t1 || !march(s, o, d, t0, t1, t, 0))
            return 0;
        v3 q = add(sub(o, s->p0), mul(d, *t));
        v3 c = V(clampd(q.x, -s->inner.x, s->inner.x), clampd(q.y, -s->inner.y, s->inner.y),
                 clampd(q.z, -s->inner.z, s->inner.z));
        *n = unit(sub(q, c));
        return 1;
    }
    case TAPER: {
        double tn = 1e-4, tf = tmax;
        int enter = -1;
        for (int k = 0; k < 10; ++k) {
            double den = dot3(s->pn[k], d), dist = s->pw[k] - dot3(s->pn[k], o);
            if (fabs(den) < 1e-15) {
                if (dist < 0)
                    return 0;
                continue;
            }
            double tt = dist / den;
            if (den < 0) {
                if (tt > tn) {
                    tn = tt;
                    enter = k;
                }
            } else if (tt < tf) {
                tf = tt;
            }
        }
        if (enter < 0 || tn > tf)
            return 0;
        *t = tn;
        *n = s->pn[enter];
        return 1;
    }
    case CYLINDER: {
        int ribbed = s->material == M_RIBS;
        double depth = ribbed ? 0.12 * s->r : 0.0, k = 2.0 * PI / 0.010;
        double rs = s->r - 0.5 * depth, best = tmax;
        int kind = -1;
        v3 rel = sub(o, s->p0);
        double zo = dot3(rel, s->axis), zd = dot3(d, s->axis);
        v3 po = sub(rel, mul(s->axis, zo)), pd = sub(d, mul(s->axis, zd));
        double A = dot3(pd, pd), B = dot3(po, pd), C = dot3(po, po) - rs * rs;
        if (A > 1e-15 && B * B - A * C >= 0) {
            double q = sqrt(B * B - A * C);
            double roots[2] = {(-B - q) / A, (-B + q) / A};
            for (int i = 0; i < 2; ++i) {
                double z = zo + zd * roots[i];
                if (roots[i] > 1e-4 && roots[i] < best && z >= 0 && z <= s->len) {
                    best = roots[i];
                    kind = 0;
                    break;
                }
            }
        }
        if (fabs(zd) > 1e-15) {
            for (int e = 0; e < 2; ++e) {
                double z = e ? s->len : 0.0, tt = (z - zo) / zd;
                v3 p = sub(add(rel, mul(d, tt)), mul(s->axis, z));
                if (tt > 1e-4 && tt < best && dot3(p, p) <= s->r * s->r) {
                    best = tt;
                    kind = 1 + e;
                }
            }
        }
        if (kind < 0)
            return 0;
        *t = best;
        if (kind == 0) {
            v3 p = add(rel, mul(d, best));
            double z = dot3(p, s->axis);
            v3 radial = unit(sub(p, mul(s->axis, z)));
            *n = unit(add(radial, mul(s->axis, ribbed ? depth * 0.5 * k * sin(k * z) : 0.0)));
        } else {
            *n = kind == 1 ? mul(s->axis, -1.0) : s->axis;
        }
        return 1;
    }
    case RING: {
        v3 oc = sub(o, s->p0);
        double R = s->r + s->r2, b = dot3(oc, d), disc = b * b - (dot3(oc, oc) - R * R);
        if (disc < 0)
            return 0;
        double t0 = fmax(-b - sqrt(disc), 1e-4), t1 = fmin(-b + sqrt(disc), tmax);
        if (t0 > t1 || !march(s, o, d, t0, t1, t, 1))
            return 0;
        v3 w = add(oc, mul(d, *t));
        double h = dot3(w, s->axis);
        v3 rad = sub(w, mul(s->axis, h));
        double rl = norm(rad);
        *n = unit(sub(w, mul(rad, rl > 1e-12 ? s->r / rl : 0.0)));
        return 1;
    }
    }
    return 0;
}

/* every column as a box [x0, x1] x [y0, y1] x [bottom, h]: nearest entry */
static int terrain_hit(const scene *S, v3 o, v3 d, double tmax, double *t, v3 *n, int *cx, int *cy)
{
    int found = 0;
    for (int iy = 0; iy < S->ny; ++iy) {
        for (int ix = 0; ix < S->nx; ++ix) {
            double lo[3] = {S->ox + ix * S->cell, S->oy + iy * S->cell, S->bottom};
            double hi[3] = {lo[0] + S->cell, lo[1] + S->cell, S->h[ix + iy * S->nx]};
            double oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
            double t0 = 0.0, t1 = tmax;
            int axis = 2, ok = 1;
            for (int a = 0; a < 3 && ok; ++a) {
                if (fabs(dd[a]) < 1e-15) {
                    ok = oo[a] >= lo[a] && oo[a] <= hi[a];
                    continue;
                }
                double ta = (lo[a] - oo[a]) / dd[a], tb = (hi[a] - oo[a]) / dd[a];
                if (ta > tb) {
                    double s = ta;
                    ta = tb;
                    tb = s;
                }
                if (ta > t0) {
                    t0 = ta;
                    axis = a;
                }
                if (tb < t1)
                    t1 = tb;
                ok = t0 <= t1;
            }
            if (!ok || t0 >= tmax)
                continue;
            tmax = t0;
            *t = t0;
            *cx = ix;
            *cy = iy;
            *n = axis == 0 ? V(d.x > 0 ? -1 : 1, 0, 0) : (axis == 1 ? V(0, d.y > 0 ? -1 : 1, 0) : V(0, 0, 1));
            found = 1;
        }
    }
    return found;
}

static int blocked(const scene *S, v3 p)
{
    double t;
    v3 n;
    int a, b;
    if (terrain_hit(S, p, S->sun, 1e9, &t, &n, &a, &b))
        return 1;
    for (int i = 0; i < S->ns; ++i) {
        const shape *s = &S->s[i];
        if (s->glow || !s->robot)
            continue;
        v3 o = mtv(s->m, sub(p, s->x)), d = mtv(s->m, S->sun);
        if (shape_hit(s, o, d, 60.0, &t, &n))
            return 1;
    }
    return 0;
}

static v3 light(v3 a, double spec, double gloss, v3 n, v3 v, v3 l, v3 c)
{
    double dd = fmax(dot3(n, l), 0.0);
    double s = pow(fmax(dot3(n, unit(add(l, v))), 0.0), gloss) * (gloss + 8.0) / 25.0;
    return V((a.x + spec * s) * dd * c.x, (a.y + spec * s) * dd * c.y, (a.z + spec * s) * dd * c.z);
}

static int to8(double x) { return (int)floor(clampd(x, 0.0, 1.0) * 255.0 + 0.5); }

/* ---- one frame: camera, lights, shapes (csrc/arc_render.c:700-716,
 * 986-1062), then every pixel. cam = {initialised, target x, y, z, heading}
 * is the camera's state, updated in place like the reference's renderer
 * updates its own. */

int oracle_render(const arc_world *w, const double *markers, int n_markers, int active, double *cam,
                  double yaw_off, double pitch, double dist, int width, int height, int samples,
                  unsigned char *rgb);

int oracle_render(const arc_world *w, const double *markers, int n_markers, int active, double *cam,
                  double yaw_off, double pitch, double dist, int width, int height, int samples,
                  unsigned char *rgb)
{
    static scene S;
    memset(&S, 0, sizeof(S));
    const arcw_terrain *tr = &w->terrain;
    S.nx = tr->nx;
    S.ny = tr->ny;
    S.cell = tr->cell;
    S.ox = tr->ox;
    S.oy = tr->oy;
    S.outside = tr->outside;
    S.h = tr->h;
    S.lo = 1e30;
    S.hi = -1e30;
    for (int k = 0; k < S.nx * S.ny; ++k) {
        S.lo = fmin(S.lo, S.h[k]);
        S.hi = fmax(S.hi, S.h[k]);
    }
    if (S.nx * S.ny == 0)
        S.lo = S.hi = 0.0;
    S.bottom = S.lo - 6.0;
    for (int k = 0; k < 9; ++k) {
        double x = S.ox + S.nx * S.cell * (k % 3 + 0.5) / 3, y = S.oy + S.ny * S.cell * (k / 3 + 0.5) / 3;
        double top = S.lo;
        for (double dx = -1.0; dx <= 1.0; dx += 0.5 * S.cell)
            for (double dy = -1.0; dy <= 1.0; dy += 0.5 * S.cell)
                top = fmax(top, height_at(&S, x + dx, y + dy));
        S.lamps[k] = V(x, y, top + 3.0);
    }
    /* camera: cam = {init, tx, ty, tz, heading} */
    const arcw_body *torso = &w->bodies[0];
    double m0[9];
    quat_mat(torso->q, m0);
    v3 fwd_b = mv(m0, V(1, 0, 0));
    double heading = atan2(fwd_b.y, fwd_b.x);
    v3 target = add(cv(torso->x), V(0, 0, 0.1));
    v3 ct = V(cam[1], cam[2], cam[3]);
    if (cam[0] == 0.0 || norm(sub(target, ct)) > 3.0) {
        ct = target;
        cam[4] = heading;
        cam[0] = 1.0;
    }
    ct = add(ct, mul(sub(target, ct), 0.15));
    double dh = heading - cam[4];
    while (dh > PI)
        dh -= 2 * PI;
    while (dh < -PI)
        dh += 2 * PI;
    cam[4] += 0.03 * dh;
    cam[1] = ct.x;
    cam[2] = ct.y;
    cam[3] = ct.z;
    double yaw = cam[4] + PI + yaw_off;
    v3 eye = add(ct, V(dist * cos(pitch) * cos(yaw), dist * cos(pitch) * sin(yaw), dist * sin(pitch)));
    eye.z = fmax(eye.z, height_at(&S, eye.x, eye.y) + 0.2);
    S.eye = eye;
    S.target = ct;
    S.fwd = unit(sub(ct, eye));
    S.right = unit(crs(S.fwd, V(0, 0, 1)));
    S.up = crs(S.right, S.fwd);
    S.tan_y = tan(25.0 * PI / 180.0);
    S.aspect = (double)width / height;
    S.fog_start = norm(sub(eye, ct));
    S.focus[0] = ct.x;
    S.focus[1] = ct.y;
    {
        float tf = (float)w->time;
        S.time_frac = tf - floorf(tf);
    }
    S.sun = unit(V(0.48, 0.30, 0.82));
    S.fill = unit(V(-0.48, -0.30, 0.45));
    {
        v3 lf = mul(S.sun, -1.0);
        S.sl = unit(crs(lf, V(0, 0, 1)));
        S.ul = crs(S.sl, lf);
        double texel = 14.0 / 2048.0;
        S.sc[0] = floor(dot3(S.sl, ct) / texel) * texel;
        S.sc[1] = floor(dot3(S.ul, ct) / texel) * texel;
    }
    /* shapes of the robot */
    S.eye_pos = V(0, 0, -100);
    S.eye_dir = V(1, 0, 0);
    S.eye_col = V(0, 0, 0);
    int eye_found = 0;
    for (int i = 0; i < w->n_visuals; ++i) {
        const arcw_visual *v = &w->visuals[i];
        shape *s = &S.s[S.ns];
        if (!shape_of(v, s))
            continue;
        s->robot = 1;
        quat_mat(w->bodies[v->body].q, s->m);
        s->x = cv(w->bodies[v->body].x);
        S.ns++;
        v3 local = v->type == CYLINDER || v->type == TAPER ? mul(add(cv(v->p0), cv(v->p1)), 0.5) : cv(v->p0);
        v3 centre = add(s->x, mv(s->m, local));
        if (!eye_found && v->material == M_GLOW && v->type == RING && v->body == 0) {
            v3 axis = mv(s->m, unit(cv(v->p1)));
            S.eye_pos = add(centre, mul(axis, 0.05));
            S.eye_dir = unit(add(axis, V(0, 0, -0.35)));
            S.eye_col = V(2.2 * v->color[0] * v->color[0], 2.2 * v->color[1] * v->color[1],
                          2.2 * v->color[2] * v->color[2]);
            eye_found = 1;
        }
        if (s->glow && S.ng < 32) {
            double sz = v->type == RING ? 1.7 * (v->radius + v->radius2) : 3.5 * v->radius;
            S.g[S.ng].c = add(centre, mul(unit(sub(eye, centre)), 0.6 * sz));
            S.g[S.ng].s = sz;
            S.g[S.ng].col = V(v->color[0], v->color[1], v->color[2]);
            S.g[S.ng].alpha = v->type == RING ? 0.4 : 0.3;
            S.g[S.ng].beam = 0;
            S.ng++;
        }
    }
    S.beacon_pos = V(0, 0, -100);
    S.beacon_col = V(0, 0, 0);
    if (!markers)
        n_markers = 0;
    if (n_markers > 4)
        n_markers = 4;
    if (n_markers > 0) {
        double k = active == 0 ? 1.6 : 0.8;
        /* the beacon colours are float constants (shader uniforms) */
        const float *cf = active == 0 ? SEEN_F : UNSEEN_F;
        S.beacon_pos = V((float)markers[0], (float)markers[1], (double)(float)markers[2] + 1.1);
        S.beacon_col = V(k * cf[0], k * cf[1], k * cf[2]);
    }
    for (int i = 0; i < n_markers; ++i) {
        const double *m = markers + 4 * i;
        double mx = (float)m[0], my = (float)m[1], mz = (float)m[2], mr = (float)m[3];
        const float *cf = i == active ? SEEN_F : UNSEEN_F;
        v3 col = V(cf[0], cf[1], cf[2]);
        v3 p = V(mx, my, mz + 1.1 + 0.06 * sin(3.0 * w->time));
        for (int e = 0; e < 2; ++e) {
            shape *s = &S.s[S.ns++];
            memset(s, 0, sizeof(*s));
            s->type = e == 0 ? SPHERE : RING;
            s->material = M_GLOW;
            s->glow = 1;
            for (int k = 0; k < 3; ++k)
                s->col[k] = sqrtf(cf[k]);
            s->m[0] = s->m[4] = s->m[8] = 1.0;
            s->x = V(0, 0, 0);
            if (e == 0) {
                s->p0 = p;
                s->r = 0.07;
            } else {
                s->p0 = V(mx, my, mz + 0.01);
                s->axis = V(0, 0, 1);
                s->r = mr;
                s->r2 = 0.012;
            }
        }
        if (S.ng + 2 <= 32) {
            S.g[S.ng].c = add(p, mul(unit(sub(eye, p)), 0.3));
            S.g[S.ng].s = 0.45;
            S.g[S.ng].col = col;
            S.g[S.ng].alpha = 0.8;
            S.g[S.ng].beam = 0;
            S.ng++;
            v3 base = V(mx, my, mz);
            S.g[S.ng].c = base;
            S.g[S.ng].side = unit(crs(V(0, 0, 1), sub(eye, base)));
            S.g[S.ng].s = 0.1;
            S.g[S.ng].col = col;
            S.g[S.ng].alpha = 0.5;
            S.g[S.ng].beam = 1;
            S.ng++;
        }
    }

    /* ---- pixels */
    static const double SP[4][2] = {{0.375, 0.125}, {0.875, 0.375}, {0.125, 0.625}, {0.625, 0.875}};
    const double sx = 2.0 / width * S.tan_y * S.aspect, sy = 2.0 / height * S.tan_y;
    for (int row = 0; row < height; ++row) {
        for (int px = 0; px < width; ++px) {
            const double wyp = height - 1 - row;
            double vx = (px + 0.5) / width - 0.5, vy = (wyp + 0.5) / height - 0.5;
            vx *= (double)width / height;
            const double vig = 1.0 - 0.4 * sstep(0.45, 1.1, sqrt(vx * vx + vy * vy));
            const double dither =
                (hash_f(fmaf(S.time_frac, 61.0f, (float)px + 0.5f), fmaf(S.time_frac, 61.0f, (float)wyp + 0.5f)) -
                 0.5) / 255.0;
            int acc[3] = {0, 0, 0};
            /* shaded once per pixel and surface (a visual, or one face of a
             * column): later samples on the same surface reuse the colour */
            long gid[4] = {-1, -1, -1, -1};
            int gcol[4][3], ngroups = 0;
            for (int si = 0; si < samples; ++si) {
                double wx = samples == 1 ? px + 0.5 : px + SP[si][0];
                double wy = samples == 1 ? wyp + 0.5 : wyp + SP[si][1];
                v3 Du = add(S.fwd, add(mul(S.right, (wx - 0.5 * width) * sx), mul(S.up, (wy - 0.5 * height) * sy)));
                v3 d = unit(Du);
                double best = 120.0 / dot3(d, S.fwd);
                int kind = -1, cx = 0, cy = 0, hit = -1;
                v3 n = V(0, 0, 1), tn;
                double t;
                if (terrain_hit(&S, eye, d, best, &t, &tn, &cx, &cy)) {
                    best = t;
                    kind = 0;
                    n = tn;
                }
                for (int i = 0; i < S.ns; ++i) {
                    const shape *s = &S.s[i];
                    v3 o = mtv(s->m, sub(eye, s->x)), dl = mtv(s->m, d);
                    if (shape_hit(s, o, dl, best, &t, &tn)) {
                        best = t;
                        kind = 1;
                        hit = i;
                        n = unit(mv(s->m, tn));
                    }
                }
                int s8[3] = {0, 0, 0};
                long sid = -1;
                if (kind == 0)
                    sid = 1000000L + (long)(cy * 64 + cx) * 8 +
                          (n.z > 0.5 ? 0 : (n.x < -0.5 ? 1 : (n.x > 0.5 ? 2 : (n.y < -0.5 ? 3 : 4))));
                else if (kind == 1)
                    sid = hit;
                int reuse = -1;
                for (int q = 0; q < ngroups; ++q)
                    if (gid[q] == sid)
                        reuse = q;
                if (reuse >= 0) {
                    for (int k = 0; k < 3; ++k)
                        s8[k] = gcol[reuse][k];
                } else if (kind >= 0) {
                    v3 p = add(eye, mul(d, best));
                    v3 alb;
                    double spec, gloss, emis, rim = 0.0, w_t = 0.0, wl = 0.0, wn = 0.0;
                    int pat;
                    v3 obj = V(0, 0, 0), o_unit = V(0, 0, 1);
                    /* neighbouring pixels' rays on the tangent plane */
                    v3 dps[2];
                    for (int k = 0; k < 2; ++k) {
                        v3 D2 = add(Du, k ? mul(S.up, sy) : mul(S.right, sx));
                        double den = dot3(D2, n);
                        dps[k] = fabs(den) > 1e-9 ? sub(add(eye, mul(D2, dot3(sub(p, eye), n) / den)), p)
                                                  : V(1e3, 1e3, 1e3);
                    }
                    if (kind == 0) {
                        double h = cell_at(&S, cx, cy);
                        double base = 0.36 + 0.05 * ((double)0) + 0.09 * clampd(h, -0.3, 0.4);
                        {
                            uint64_t hh = (uint64_t)((int64_t)cx * 73856093LL) ^ (uint64_t)((int64_t)cy * 19349663LL);
                            hh = (hh ^ (hh >> 13)) * 1274126177ULL;
                            base += 0.05 * (double)((hh >> 8) & 0xffff) / 65535.0;
                        }
                        double c;
                        if (n.z > 0.5) {
                            double occ[4], cq[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
                            for (int q = 0; q < 4; ++q) {
                                int qx = (int)cq[q][0], qy = (int)cq[q][1];
                                double a = clampd((cell_at(&S, cx + qx, cy) - h) / 0.12, 0, 1);
                                double b = clampd((cell_at(&S, cx, cy + qy) - h) / 0.12, 0, 1);
                                double e = clampd((cell_at(&S, cx + qx, cy + qy) - h) / 0.12, 0, 1);
                                occ[q] = base * (1.0 - 0.22 * (a + b + 0.5 * e));
                            }
                            double u = clampd((p.x - (S.ox + cx * S.cell)) / S.cell, 0, 1);
                            double v = clampd((p.y - (S.oy + cy * S.cell)) / S.cell, 0, 1);
                            c = u >= v ? occ[0] + u * (occ[1] - occ[0]) + v * (occ[2] - occ[1])
                                       : occ[0] + v * (occ[3] - occ[0]) + u * (occ[2] - occ[3]);
                            alb = V(c * c, c * c, 1.04 * c * 1.04 * c);
                        } else {
                            double cs = 0.8 * base;
                            int ax = cx + (n.x > 0.5 ? 1 : (n.x < -0.5 ? -1 : 0));
                            int ay = cy + (n.y > 0.5 ? 1 : (n.y < -0.5 ? -1 : 0));
                            double zlo = fmax(cell_at(&S, ax, ay), S.bottom);
                            double f = h > zlo ? clampd((p.z - zlo) / (h - zlo), 0, 1) : 1.0;
                            v3 col = V(lerp(0.45 * cs, cs, f), lerp(0.45 * cs, cs, f), lerp(0.47 * cs, 1.04 * cs, f));
                            alb = hadamard(col, col);
                        }
                        spec = 0.25;
                        gloss = 16.0;
                        emis = 0.0;
                        pat = 1;
                        for (int k = 0; k < 2; ++k)
                            w_t += (fabs(dps[k].x) + fabs(dps[k].y)) / S.cell;
                    } else {
                        const shape *s = &S.s[hit];
                        alb = V(s->col[0] * s->col[0], s->col[1] * s->col[1], s->col[2] * s->col[2]);
                        spec = MAT[s->material][0];
                        gloss = MAT[s->material][1];
                        emis = MAT[s->material][2];
                        pat = (int)MAT[s->material][3];
                        rim = s->robot ? 1.0 : 0.0;
                        v3 pl = mtv(s->m, sub(p, s->x));
                        obj = s->type == SPHERE ? mul(sub(pl, s->p0), 1.0 / s->r) : pl;
                        if (pat == 2) {
                            o_unit = unit(obj);
                            double ct_ = sqrt(fmax(1.0 - o_unit.z * o_unit.z, 1e-12));
                            double rxy = fmax(o_unit.x * o_unit.x + o_unit.y * o_unit.y, 1e-12);
                            for (int k = 0; k < 2; ++k) {
                                v3 dob = mul(mtv(s->m, dps[k]), 1.0 / s->r);
                                wl += fabs(dob.z / ct_) * 7.0 / 3.14159;
                                wn += fabs((o_unit.x * dob.y - o_unit.y * dob.x) / rxy) * 6.0 / 3.14159;
                            }
                        }
                    }
                    /* the shader */
                    v3 v = unit(sub(eye, p)), a = alb;
                    if (pat == 1) {
                        double gx = (p.x - S.ox) / S.cell, gy = (p.y - S.oy) / S.cell;
                        double fx = 0.5 - fabs(fract_d(gx) - 0.5), fy = 0.5 - fabs(fract_d(gy) - 0.5);
                        double grime = 0.6 * vnoise(p.x * 1.7, p.y * 1.7) + 0.4 * vnoise(p.x * 6 + p.z * 4, p.y * 6 + p.z * 4);
                        a = mul(a, lerp(0.65, 1.25, grime));
                        if (n.z > 0.7)
                            a = mul(a, lerp(0.35, 1.0, sstep(0.0, 0.02 + w_t, fmin(fx, fy))));
                        spec *= grime;
                        rim = 0.0;
                    } else if (pat == 2) {
                        double lat = asin(clampd(o_unit.z, -1, 1)) * 7.0 / 3.14159;
                        double lon = atan2(o_unit.y, o_unit.x) * 6.0 / 3.14159 + 0.5 * floor(lat);
                        double s1 = 1.0 - sstep(0.0, 0.04 + 1.2 * wl, 0.5 - fabs(fract_d(lat) - 0.5));
                        double s2 = (1.0 - sstep(0.0, 0.03 + 1.2 * wn, 0.5 - fabs(fract_d(lon) - 0.5))) *
                                    (fabs(o_unit.z) <= 0.92 ? 1.0 : 0.0);
                        double mm = fmax(s1, s2);
                        a = mul(a, 1.0 - 0.7 * mm);
                        spec *= 1.0 - 0.8 * mm;
                    }
                    if (rim > 0.5) {
                        double wear = 0.6 * vnoise(obj.x * 30 + obj.z * 17, obj.y * 30 + obj.z * 17) +
                                      0.4 * vnoise(obj.y * 90 + obj.x * 41, obj.z * 90 + obj.x * 41);
                        a = mul(a, lerp(0.7, 1.15, wear));
                        spec *= lerp(0.4, 1.4, wear);
                    }
                    double hemi = 0.5 + 0.5 * n.z;
                    v3 c = hadamard(a, V(lerp(GND[0], SKY[0], hemi), lerp(GND[1], SKY[1], hemi), lerp(GND[2], SKY[2], hemi)));
                    double qx = (p.x - S.focus[0]) / 6.0, qy = (p.y - S.focus[1]) / 6.0;
                    double pool = 0.65 + 0.35 * exp(-(qx * qx + qy * qy));
                    v3 pb = add(p, mul(n, 3.0 * 7.0 / 2048.0));
                    double ex = fabs(dot3(pb, S.sl) - S.sc[0]) / 14.0, ey = fabs(dot3(pb, S.ul) - S.sc[1]) / 14.0;
                    double fade = sstep(0.5, 0.42, fmax(ex, ey));
                    double k_lit = 1.0;
                    if (fade > 0.0 && dot3(n, S.sun) > 0.0)
                        k_lit = lerp(1.0, blocked(&S, add(p, mul(n, 2e-3))) ? 0.0 : 1.0, fade);
                    c = add(c, mul(light(a, spec, gloss, n, v, S.sun, V(SUN_C[0], SUN_C[1], SUN_C[2])), k_lit * pool));
                    c = add(c, light(a, spec, gloss, n, v, S.fill, V(FILL_C[0], FILL_C[1], FILL_C[2])));
                    for (int i = 0; i < 9; ++i) {
                        v3 l = sub(S.lamps[i], p);
                        double d2 = dot3(l, l);
                        if (d2 > 64.0)
                            continue;
                        l = mul(l, 1.0 / sqrt(d2));
                        c = add(c, mul(light(a, spec, gloss, n, v, l, V(LAMP_C[0], LAMP_C[1], LAMP_C[2])),
                                       sstep(0.25, 0.8, l.z) / (1.0 + 0.12 * d2)));
                    }
                    {
                        v3 l = sub(S.eye_pos, p);
                        double d2 = dot3(l, l);
                        l = mul(l, 1.0 / sqrt(d2));
                        double cone = sstep(0.35, 0.85, -dot3(l, S.eye_dir));
                        c = add(c, mul(light(a, spec, gloss, n, v, l, S.eye_col), cone / (1.0 + 2.0 * d2)));
                    }
                    {
                        v3 l = sub(S.beacon_pos, p);
                        double d2 = dot3(l, l);
                        c = add(c, mul(light(a, spec, gloss, n, v, mul(l, 1.0 / sqrt(d2)), S.beacon_col),
                                       1.0 / (1.0 + 1.5 * d2)));
                    }
                    double nv = 1.0 - fmax(dot3(n, v), 0.0);
                    v3 r = sub(mul(n, 2.0 * dot3(n, v)), v);
                    double hr = 0.5 + 0.5 * r.z, shn = spec * (0.04 + 0.5 * pow(nv, 5.0));
                    c = add(c, V(shn * lerp(GND[0], 3 * SKY[0], hr), shn * lerp(GND[1], 3 * SKY[1], hr),
                                 shn * lerp(GND[2], 3 * SKY[2], hr)));
                    c = add(c, mul(V(SKY[0], SKY[1], SKY[2]), rim * pow(nv, 4.0) * 0.6));
                    if (emis >= 0.5)
                        c = mul(a, emis);
                    c = mul(c, exp(-0.05 * fmax(norm(sub(eye, p)) - S.fog_start, 0.0)));
                    c = mul(c, sstep(S.lo - 3.0, S.lo + 0.2, p.z));
                    double cc[3] = {c.x, c.y, c.z};
                    for (int k = 0; k < 3; ++k) {
                        double x = cc[k];
                        x = x * (2.51 * x + 0.03) / (x * (2.43 * x + 0.59) + 0.14);
                        s8[k] = to8(pow(clampd(x, 0, 1), 1.0 / 2.2) + dither);
                    }
                    if (ngroups < 4) {
                        gid[ngroups] = sid;
                        for (int k = 0; k < 3; ++k)
                            gcol[ngroups][k] = s8[k];
                        ngroups++;
                    }
                }
                /* glow, depth tested against the scene */
                double tdepth = kind >= 0 ? best : 1e30;
                v3 g = V(0, 0, 0);
                for (int i = 0; i < S.ng; ++i) {
                    double tt, u, vv, k;
                    if (!S.g[i].beam) {
                        double den = dot3(d, S.fwd);
                        if (den <= 1e-6)
                            continue;
                        tt = dot3(sub(S.g[i].c, eye), S.fwd) / den;
                        if (tt <= 0 || tt >= tdepth)
                            continue;
                        v3 q = sub(add(eye, mul(d, tt)), S.g[i].c);
                        u = dot3(q, S.right) / S.g[i].s;
                        vv = dot3(q, S.up) / S.g[i].s;
                        if (fabs(u) > 1 || fabs(vv) > 1)
                            continue;
                        double r2 = u * u + vv * vv;
                        k = (exp(-6 * r2) * 0.8 + exp(-30 * r2)) * (1.0 - sstep(0.7, 1.0, r2));
                    } else {
                        v3 nb = crs(S.g[i].side, V(0, 0, 1));
                        double den = dot3(d, nb);
                        if (fabs(den) <= 1e-9)
                            continue;
                        tt = dot3(sub(S.g[i].c, eye), nb) / den;
                        if (tt <= 0 || tt >= tdepth)
                            continue;
                        v3 q = sub(add(eye, mul(d, tt)), S.g[i].c);
                        u = dot3(q, S.g[i].side) / S.g[i].s;
                        vv = q.z / 3.5;
                        if (fabs(u) > 1 || vv < 0 || vv > 1)
                            continue;
                        k = exp(-12 * u * u) * (1 - vv) * (1 - vv);
                    }
                    v3 P = add(eye, mul(d, tt));
                    k *= S.g[i].alpha * exp(-0.05 * fmax(norm(sub(eye, P)) - S.fog_start, 0.0));
                    g = add(g, mul(S.g[i].col, k));
                }
                double gg[3] = {g.x, g.y, g.z};
                for (int k = 0; k < 3; ++k)
                    acc[k] += (int)floor(to8(s8[k] / 255.0 + gg[k]) * vig + 0.5);
            }
            unsigned char *o = rgb + ((size_t)row * width + px) * 3;
            for (int k = 0; k < 3; ++k)
                o[k] = (unsigned char)((acc[k] + samples / 2) / samples);
        }
    }
    return 0;
}
