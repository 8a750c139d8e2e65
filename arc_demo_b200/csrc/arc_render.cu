// arc_render.cu - headless renderer: the worlds of an arc_sim ray cast into
// RGB frames on the GPU, behind the ABI of include/arc_render.h.
//
// The reference draws one world with OpenGL 2.1 (csrc/arc_render.c,
// csrc/arc_mesh.c): tessellated meshes of the robot's visuals and of the
// block terrain, one GLSL shader for all lighting, a shadow map, additive
// glow billboards, a vignette and 4x multisampling. Here the same scene is
// ray cast, any number of worlds per launch:
//
//   k_frame_setup  one warp per rendered world: the camera (the
//                  reference's smoothed orbit behind the robot, one state
//                  per world), the lights, the world pose of every body,
//                  the markers and glow billboards, the terrain's lowest
//                  and highest column and the lamp heights above it.
//   k_render       one CTA per 16 x 16 pixel tile of one world: the tile's
//                  frustum culls the visuals' bounding spheres into a list
//                  in shared memory; each thread traces its pixel's samples
//                  (the terrain by a 2D DDA over the columns, the visuals
//                  exactly or by sphere tracing), shades them with the
//                  reference's shader, adds the glow, applies the vignette
//                  and averages the samples.
//
// Departures from the rasteriser, all in fine detail: shapes are exact
// (spheres, capped cylinders, chamfered prisms) or sphere traced (rounded
// boxes, tori) where the reference tessellates them; the key light's shadow
// is one ray toward the sun where the reference filters four taps of a
// 2048^2 shadow map; like multisampling, a pixel is shaded once per surface
// its samples hit, but at the first such sample's hit point rather than at
// the pixel centre, and a surface is a whole visual or column face rather
// than one triangle of it; the screen-space derivatives of the shader
// (fwidth) come from ray differentials; the terrain's top quads are split
// along the diagonal from their (-x, -y) corner for the interpolation of
// the vertex colours.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "arc_model.h"
#include "arc_task.cuh"
#include "../../include/arc_render.h"

// CTAs of k_render resident per SM. 4 caps its registers at 64 at the cost
// of ~250 bytes of spills to L1; the extra warps hide more latency than the
// spills cost (ms per 256 frames of 640 x 360 x 4 rays: 2 CTAs 24.7, 3 20.6,
// 4 20.0).
#ifndef ARC_RENDER_MIN_BLOCKS
#define ARC_RENDER_MIN_BLOCKS 4
#endif

namespace arc {
namespace rd {

using F3 = V3<float>;

constexpr int kTileW = 16, kTileH = 16, kThreads = kTileW * kTileH;
constexpr int kMaxMarkers = 4;
constexpr int kLampGrid = 3, kLamps = kLampGrid * kLampGrid;  // csrc/arc_render.c:36-38
constexpr int kPoses = kMaxBodies + 1;                          // + the identity pose of world-frame items
constexpr int kIdentity = kMaxBodies;
constexpr int kMaxItems = kMaxVisuals + 2 * kMaxMarkers;
constexpr int kMaxGlow = 16 + 2 * kMaxMarkers;
constexpr float kFar = 120.0f;                                  // csrc/arc_render.c:1058
constexpr double kShadowRange = 7.0;                            // csrc/arc_render.c:33
constexpr double kShadowTexel = 2.0 * kShadowRange / 2048.0;
constexpr float kShadowNormalOffset = (float)(3.0 * kShadowRange / 2048.0);
constexpr double kVoidDepth = 6.0, kLampHeight = 3.0, kBeaconHeight = 1.1;
constexpr float kFogDensity = 0.05f;

// The look (csrc/arc_render.c:93-117): linear colours.
__constant__ float c_sun_col[3] = {1.45f, 1.55f, 1.80f};
__constant__ float c_fill_col[3] = {0.16f, 0.13f, 0.11f};
__constant__ float c_lamp_col[3] = {0.40f, 0.30f, 0.20f};
__constant__ float c_sky[3] = {0.090f, 0.100f, 0.125f};
__constant__ float c_gnd[3] = {0.030f, 0.030f, 0.034f};
// per material: specular, glossiness, emission, pattern (1 terrain, 2 panels)
__constant__ float c_mat[7][4] = {
    {0.45f, 36.0f, 0.0f, 0.0f},  {0.50f, 40.0f, 0.0f, 2.0f}, {0.90f, 64.0f, 0.0f, 0.0f}, {0.08f, 10.0f, 0.0f, 0.0f},
    {1.80f, 180.0f, 0.0f, 0.0f}, {0.60f, 40.0f, 0.0f, 0.0f}, {0.00f, 1.0f, 3.0f, 0.0f}};
constexpr double kSunDir[3] = {0.48, 0.30, 0.82}, kFillDir[3] = {-0.48, -0.30, 0.45};
constexpr double kEyeLight = 2.2;
__constant__ float c_beacon_seen[3] = {1.00f, 0.42f, 0.08f}, c_beacon_unseen[3] = {0.20f, 0.55f, 1.00f};

// One visual ready for intersection, in its body's frame.
//   sphere    o centre, a radius
//   box       o centre, (a, b, c) inner half extents, e bevel radius
//   taper     pl: ten planes n.x <= w (eight chamfered sides, two caps)
//   cylinder  o = p0, d axis, a radius, b length, c rib depth, e rib wavenumber
//   ring      o centre, d axis, a major radius, b tube radius
struct VisK {
    int type, body, material, glow;
    float col[3], rim;
    float bc[3], br;  // bounding sphere
    float o[3], a;
    float d[3], b;
    float c, e, pad0, pad1;
    float pl[10][4];
};

struct GlowK {       // an additive billboard (csrc/arc_render.c:625-672)
    float c[3], s;   // halo: centre and half size; beam: base and half width
    float col[3], alpha;
    float side[3];   // beam: its horizontal direction
    int beam;
};

struct FrameK {
    float eye[3], fwd[3], right[3], up[3];
    float tan_y, aspect, fog_start, time;
    float floor_z, bottom, hmax, pad0;
    float focus[2], shadow_c[2];
    float sun[3], fill[3], sl[3], ul[3];
    float lamps[kLamps][3];
    float eye_pos[3], eye_dir[3], eye_col[3];
    float beacon_pos[3], beacon_col[3];
    float robot_c[3], robot_r;
    float pos[kPoses][3];
    float rot[kPoses][9];  // row major: world = rot * local + pos
    int nx, ny, n_items, n_glow;
    float cell, ox, oy, outside;
    float body_c[kPoses][3], body_r[kPoses];  // world bounding sphere of each body's shadow casters
    VisK extra[2 * kMaxMarkers];  // marker beacons and rings, world frame
    GlowK glow[kMaxGlow];
};

struct CamState {
    double target[3], heading;
    int init, pad;
};

struct CamParams {
    double yaw, pitch, dist;
    int width, height;
};

__device__ __forceinline__ F3 ld3(const float* p) { return F3{p[0], p[1], p[2]}; }
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ float mixf(float a, float b, float t) { return a + (b - a) * t; }
__device__ __forceinline__ float fractf(float x) { return x - floorf(x); }
// GLSL smoothstep, also with edge0 > edge1 (the shadow fade uses that)
__device__ __forceinline__ float smooth(float e0, float e1, float x)
{
    float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}
__device__ __forceinline__ F3 rot_mul(const float* m, F3 v)
{
    return F3{m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z,
              m[6] * v.x + m[7] * v.y + m[8] * v.z};
}
__device__ __forceinline__ F3 rot_tmul(const float* m, F3 v)
{
    return F3{m[0] * v.x + m[3] * v.y + m[6] * v.z, m[1] * v.x + m[4] * v.y + m[7] * v.z,
              m[2] * v.x + m[5] * v.y + m[8] * v.z};
}

// The shader's value noise (csrc/arc_render.c:151-158). The hash of a
// lattice point is evaluated with one rounding order (an explicit fma), so
// that CPU restatements can reproduce it. noise2, hit_visual,
// trace_terrain and shade_light stay out of line and the taper's plane loop
// stays rolled: the kernel's code is larger than the instruction cache, and
// one copy of each is faster than inlined copies. For the same reason this
// file is compiled with the approximate (at most 2 ulp) division and square
// root, whose code is a fraction of the IEEE versions'.
__device__ __noinline__ float hash2(float x, float y)
{
    return fractf(__fmul_rn(sinf(fmaf(x, 127.1f, y * 311.7f)), 43758.5453f));
}
__device__ __noinline__ float noise2(float x, float y)
{
    float ix = floorf(x), iy = floorf(y);
    float fx = x - ix, fy = y - iy;
    fx = fx * fx * (3.0f - 2.0f * fx);
    fy = fy * fy * (3.0f - 2.0f * fy);
    float a = mixf(hash2(ix, iy), hash2(ix + 1.0f, iy), fx);
    float b = mixf(hash2(ix, iy + 1.0f), hash2(ix + 1.0f, iy + 1.0f), fx);
    return mixf(a, b, fy);
}

// Shade of the top of column (ix, iy) (csrc/arc_mesh.c:194-200).
__device__ __forceinline__ double cell_hash(int ix, int iy)
{
    unsigned long long h = (unsigned long long)((long long)ix * 73856093LL) ^
                           (unsigned long long)((long long)iy * 19349663LL);
    h = (h ^ (h >> 13)) * 1274126177ULL;
    return (double)((h >> 8) & 0xffff) / 65535.0;
}

template <class R> struct TerrainF {
    const R* h;
    int nx, ny;
    float cell, ox, oy, outside, hmax, bottom;
    __device__ __forceinline__ float at(int ix, int iy) const
    {
        if (ix < 0 || iy < 0 || ix >= nx || iy >= ny)
            return outside;
        return (float)h[ix + iy * nx];
    }
};

enum Face { kFaceTop = 0, kFaceX = 1, kFaceY = 2 };

// First column surface along o + t D, t in (0, tmax): the drawn surface of
// csrc/arc_mesh.c:228-255 (column tops, and column sides where the
// neighbour is lower, down to the void's bottom). A 2D DDA over the cells
// the ray crosses inside the grid's box. Returns t or -1.
template <class R>
__device__ __noinline__ float trace_terrain(const TerrainF<R>& T, F3 o, F3 D, float tmax, int& face, int& cx, int& cy, int& sgn)
{
    if (T.nx <= 0 || T.ny <= 0)
        return -1.0f;
    const float lo[3] = {T.ox, T.oy, T.bottom};
    const float hi[3] = {T.ox + T.nx * T.cell, T.oy + T.ny * T.cell, T.hmax};
    const float oo[3] = {o.x, o.y, o.z}, dd[3] = {D.x, D.y, D.z};
    float t0 = 0.0f, t1 = tmax;
    int entry = -1;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (fabsf(dd[a]) < 1e-12f) {
            if (oo[a] < lo[a] || oo[a] > hi[a])
                return -1.0f;
            continue;
        }
        float inv = 1.0f / dd[a];
        float ta = (lo[a] - oo[a]) * inv, tb = (hi[a] - oo[a]) * inv;
        if (ta > tb) {
            float s = ta;
            ta = tb;
            tb = s;
        }
        if (ta > t0) {
            t0 = ta;
            entry = a;
        }
        t1 = fminf(t1, tb);
    }
    if (t0 > t1)
        return -1.0f;
    const float px = o.x + D.x * t0, py = o.y + D.y * t0;
    int ix = min(max((int)floorf((px - T.ox) / T.cell), 0), T.nx - 1);
    int iy = min(max((int)floorf((py - T.oy) / T.cell), 0), T.ny - 1);
    const int sx = D.x > 0.0f ? 1 : -1, sy = D.y > 0.0f ? 1 : -1;
    const float big = 1e30f;
    const bool mx = fabsf(D.x) > 1e-12f, my = fabsf(D.y) > 1e-12f;
    const float inx = mx ? 1.0f / D.x : 0.0f, iny = my ? 1.0f / D.y : 0.0f;
    const float tdx = mx ? T.cell * fabsf(inx) : big, tdy = my ? T.cell * fabsf(iny) : big;
    float tx = mx ? (T.ox + (ix + (sx > 0)) * T.cell - o.x) * inx : big;
    float ty = my ? (T.oy + (iy + (sy > 0)) * T.cell - o.y) * iny : big;
    float t_in = t0;
    int f_in = entry == 0 ? kFaceX : (entry == 1 ? kFaceY : kFaceTop);
    int s_in = entry == 0 ? sx : sy;
    const int max_steps = T.nx + T.ny + 2;
    for (int step = 0; step < max_steps; ++step) {
        const float h = T.at(ix, iy);
        const float t_out = fminf(fminf(tx, ty), t1);
        if (o.z + D.z * t_in <= h) {
            face = f_in;
            sgn = s_in;
            cx = ix;
            cy = iy;
            return t_in;
        }
        if (D.z < 0.0f) {
            const float tt = (h - o.z) / D.z;
            if (tt <= t_out) {
                face = kFaceTop;
                sgn = 0;
                cx = ix;
                cy = iy;
                return tt;
            }
        }
        if (t_out >= t1)
            break;
        if (tx < ty) {
            ix += sx;
            t_in = tx;
            tx += tdx;
            f_in = kFaceX;
            s_in = sx;
        } else {
            iy += sy;
            t_in = ty;
            ty += tdy;
            f_in = kFaceY;
            s_in = sy;
        }
        if (ix < 0 || iy < 0 || ix >= T.nx || iy >= T.ny)
            break;
    }
    return -1.0f;
}

// ---- visuals, in their body's frame; D is a unit vector, hits in (tmin, tmax)

__device__ __forceinline__ bool hit_sphere(F3 c, float r, F3 o, F3 D, float tmin, float tmax, float& t)
{
    F3 oc = o - c;
    float b = dot(oc, D), cc = dot(oc, oc) - r * r;
    float disc = b * b - cc;
    if (disc < 0.0f)
        return false;
    float s = sqrtf(disc);
    float ta = -b - s;
    if (ta <= tmin)
        ta = -b + s;
    if (ta <= tmin || ta >= tmax)
        return false;
    t = ta;
    return true;
}

__device__ __forceinline__ float sdf_box(F3 q, F3 in, float bevel)
{
    float ax = fabsf(q.x) - in.x, ay = fabsf(q.y) - in.y, az = fabsf(q.z) - in.z;
    float ox = fmaxf(ax, 0.0f), oy = fmaxf(ay, 0.0f), oz = fmaxf(az, 0.0f);
    return sqrtf(ox * ox + oy * oy + oz * oz) + fminf(fmaxf(ax, fmaxf(ay, az)), 0.0f) - bevel;
}

__device__ __forceinline__ float sdf_ring(F3 w, F3 d, float major, float tube)
{
    float h = dot(w, d);
    F3 rad = w - scale(d, h);
    float rr = sqrtf(dot(rad, rad)) - major;
    return sqrtf(rr * rr + h * h) - tube;
}

constexpr int kMarch = 48;
constexpr float kMarchEps = 2e-5f;

__device__ __noinline__ bool hit_visual(const VisK& v, F3 o, F3 D, float tmax, float& t, F3& n)
{
    const F3 c = ld3(v.o), d = ld3(v.d);
    switch (v.type) {
    case kVisSphere: {
        if (!hit_sphere(c, v.a, o, D, 1e-4f, tmax, t))
            return false;
        n = scale(o + scale(D, t) - c, 1.0f / v.a);
        return true;
    }
    case kVisBox: {
        const F3 in{v.a, v.b, v.c};
        const float oa[3] = {o.x - c.x, o.y - c.y, o.z - c.z}, da[3] = {D.x, D.y, D.z};
        const float ext[3] = {v.a + v.e, v.b + v.e, v.c + v.e};
        float t0 = 1e-4f, t1 = tmax;
        for (int a = 0; a < 3; ++a) {
            if (fabsf(da[a]) < 1e-12f) {
                if (fabsf(oa[a]) > ext[a])
                    return false;
                continue;
            }
            float inv = 1.0f / da[a];
            float ta = (-ext[a] - oa[a]) * inv, tb = (ext[a] - oa[a]) * inv;
            t0 = fmaxf(t0, fminf(ta, tb));
            t1 = fminf(t1, fmaxf(ta, tb));
        }
        if (t0 > t1)
            return false;
        const F3 q0{oa[0], oa[1], oa[2]};
        float tt = t0;
        for (int i = 0; i < kMarch; ++i) {
            F3 q = q0 + scale(D, tt);
            float dist = sdf_box(q, in, v.e);
            if (dist < kMarchEps) {
                t = tt;
                F3 cl{clampf(q.x, -in.x, in.x), clampf(q.y, -in.y, in.y), clampf(q.z, -in.z, in.z)};
                n = normalize(q - cl);
                return true;
            }
            tt += dist;
            if (tt > t1)
                return false;
        }
        return false;
    }
    case kVisTaper: {
        float tn = 1e-4f, tf = tmax;
        int enter = -1;
#pragma unroll 1
        for (int k = 0; k < 10; ++k) {
            const F3 pn{v.pl[k][0], v.pl[k][1], v.pl[k][2]};
            float den = dot(pn, D), dist = v.pl[k][3] - dot(pn, o);
            if (fabsf(den) < 1e-12f) {
                if (dist < 0.0f)
                    return false;
                continue;
            }
            float tt = dist / den;
            if (den < 0.0f) {
                if (tt > tn) {
                    tn = tt;
                    enter = k;
                }
            } else {
                tf = fminf(tf, tt);
            }
        }
        if (enter < 0 || tn > tf)
            return false;
        t = tn;
        n = F3{v.pl[enter][0], v.pl[enter][1], v.pl[enter][2]};
        return true;
    }
    case kVisCylinder: {
        const float radius = v.a, len_ = v.b, rib = v.c;
        const float side_r = radius - 0.5f * rib;
        const F3 w = o - c;
        const float wd = dot(w, d), Dd = dot(D, d);
        const F3 a = D - scale(d, Dd), b0 = w - scale(d, wd);
        float best = tmax;
        int kind = -1;
        const float A = dot(a, a);
        if (A > 1e-12f) {
            float B = dot(a, b0), C = dot(b0, b0) - side_r * side_r;
            float disc = B * B - A * C;
            if (disc >= 0.0f) {
                float s = sqrtf(disc);
                float r0 = (-B - s) / A, r1 = (-B + s) / A;
                float z0 = wd + Dd * r0, z1 = wd + Dd * r1;
                if (r0 > 1e-4f && r0 < best && z0 >= 0.0f && z0 <= len_) {
                    best = r0;
                    kind = 0;
                } else if (r1 > 1e-4f && r1 < best && z1 >= 0.0f && z1 <= len_) {
                    best = r1;
                    kind = 0;
                }
            }
        }
        if (fabsf(Dd) > 1e-12f) {
            for (int e = 0; e < 2; ++e) {
                float z = e ? len_ : 0.0f;
                float tt = (z - wd) / Dd;
                if (tt > 1e-4f && tt < best) {
                    F3 p = w + scale(D, tt) - scale(d, z);
                    if (dot(p, p) <= radius * radius) {
                        best = tt;
                        kind = 1 + e;
                    }
                }
            }
        }
        if (kind < 0)
            return false;
        t = best;
        if (kind == 0) {
            F3 p = w + scale(D, t);
            float z = dot(p, d);
            F3 radial = normalize(p - scale(d, z));
            // ribbed sleeve: the corrugation's slope (csrc/arc_mesh.c:84-90)
            float slope = rib > 0.0f ? rib * 0.5f * (3.14159265f * v.e) * sinpif(v.e * z) : 0.0f;
            n = normalize(radial + scale(d, slope));
        } else {
            n = kind == 1 ? -d : d;
        }
        return true;
    }
    case kVisRing: {
        float t0, t1b;
        {
            F3 oc = o - c;
            float b = dot(oc, D), r = v.a + v.b, cc = dot(oc, oc) - r * r;
            float disc = b * b - cc;
            if (disc < 0.0f)
                return false;
            float s = sqrtf(disc);
            t0 = fmaxf(-b - s, 1e-4f);
            t1b = fminf(-b + s, tmax);
            if (t0 > t1b)
                return false;
        }
        const F3 w0 = o - c;
        float tt = t0;
        for (int i = 0; i < kMarch; ++i) {
            F3 w = w0 + scale(D, tt);
            float dist = sdf_ring(w, d, v.a, v.b);
            if (dist < kMarchEps) {
                t = tt;
                float h = dot(w, d);
                F3 rad = w - scale(d, h);
                float rl = sqrtf(dot(rad, rad));
                n = normalize(w - scale(rad, rl > 1e-12f ? v.a / rl : 0.0f));
                return true;
            }
            tt += dist;
            if (tt > t1b)
                return false;
        }
        return false;
    }
    }
    return false;
}

// Is the segment from p toward the sun blocked by a column or by a visual
// that casts shadows (all but the glowing ones, csrc/arc_render.c:545-552)?
template <class R>
__device__ bool shadowed(const FrameK& fr, const TerrainF<R>& T, const VisK* __restrict__ vis, int nv, F3 p)
{
    const F3 L = ld3(fr.sun);
    int f, a, b, s;
    if (trace_terrain(T, p, L, 60.0f, f, a, b, s) >= 0.0f)
        return true;
    // the robot's bounding sphere first
    F3 oc = p - ld3(fr.robot_c);
    float bb = dot(oc, L), cc = dot(oc, oc) - fr.robot_r * fr.robot_r;
    if (bb * bb - cc < 0.0f || (bb > 0.0f && cc > 0.0f))
        return false;
    // bodies whose casters' bounding sphere the ray meets
    unsigned bodies = 0u;
    for (int b = 0; b < kMaxBodies; ++b) {
        F3 q = p - ld3(fr.body_c[b]);
        float qb = dot(q, L), qc = dot(q, q) - fr.body_r[b] * fr.body_r[b];
        if (fr.body_r[b] > 0.0f && qb * qb - qc >= 0.0f && !(qb > 0.0f && qc > 0.0f))
            bodies |= 1u << b;
    }
    int last_body = -1;
    F3 ol{0, 0, 0}, dl{0, 0, 0};
    for (int i = 0; i < nv; ++i) {
        if (vis[i].glow || vis[i].type < 0 || !((bodies >> vis[i].body) & 1u))
            continue;
        const int body = vis[i].body;
        // bounding sphere in the world
        F3 cw = rot_mul(fr.rot[body], ld3(vis[i].bc)) + ld3(fr.pos[body]);
        F3 q = p - cw;
        float qb = dot(q, L), qc = dot(q, q) - vis[i].br * vis[i].br;
        if (qb * qb - qc < 0.0f || (qb > 0.0f && qc > 0.0f))
            continue;
        if (body != last_body) {
            last_body = body;
            ol = rot_tmul(fr.rot[body], p - ld3(fr.pos[body]));
            dl = rot_tmul(fr.rot[body], L);
        }
        float t;
        F3 n;
        if (hit_visual(vis[i], ol, dl, 60.0f, t, n))
            return true;
    }
    return false;
}

struct Surface {
    F3 p, n, albedo;  // albedo: the vertex colour squared
    float spec, gloss, emis, rim;
    int pat;          // 1 terrain, 2 panels
    float fw0, fw1;   // terrain: fwidth(g.x) + fwidth(g.y); panels: fwidth(lat), fwidth(lon)
    F3 obj;           // object-space position (v_obj)
    F3 g;             // terrain: grid coordinates (g.x, g.y); panels: unit-sphere point
};

// x^y for x in [0, 1], y > 0, by the hardware base-2 exponential and
// logarithm (relative error ~1e-6: far below one level of 8-bit colour);
// 0^y = 0.
__device__ __forceinline__ float pow_approx(float x, float y) { return x > 0.0f ? exp2f(y * __log2f(x)) : 0.0f; }

__device__ __noinline__ F3 shade_light(F3 a, float spec, float gloss, F3 n, F3 v, F3 l, F3 col)
{
    float d = fmaxf(dot(n, l), 0.0f);
    F3 hv = normalize(l + v);
    float s = pow_approx(fmaxf(dot(n, hv), 0.0f), gloss) * (gloss + 8.0f) / 25.0f;
    return F3{(a.x + spec * s) * d * col.x, (a.y + spec * s) * d * col.y, (a.z + spec * s) * d * col.z};
}

// The scene fragment shader (csrc/arc_render.c:159-263), up to the dither;
// `lit` is the key light's visibility.
__device__ F3 shade_scene(const FrameK& fr, const Surface& s, float lit_k)
{
    const F3 n = s.n, v = normalize(ld3(fr.eye) - s.p);
    F3 a = s.albedo;
    float spec = s.spec, gloss = s.gloss, rim = s.rim;
    if (s.pat == 1) {
        float fx = 0.5f - fabsf(fractf(s.g.x) - 0.5f), fy = 0.5f - fabsf(fractf(s.g.y) - 0.5f);
        float edge = fminf(fx, fy), w = s.fw0;
        float grime = 0.6f * noise2(s.p.x * 1.7f, s.p.y * 1.7f) +
                      0.4f * noise2(s.p.x * 6.0f + s.p.z * 4.0f, s.p.y * 6.0f + s.p.z * 4.0f);
        a = scale(a, mixf(0.65f, 1.25f, grime));
        if (n.z > 0.7f)
            a = scale(a, mixf(0.35f, 1.0f, smooth(0.0f, 0.02f + w, edge)));
        spec *= grime;
        rim = 0.0f;
    } else if (s.pat == 2) {
        const F3 o = s.g;
        float lat = asinf(clampf(o.z, -1.0f, 1.0f)) * 7.0f / 3.14159f;
        float lon = atan2f(o.y, o.x) * 6.0f / 3.14159f + 0.5f * floorf(lat);
        float wl = s.fw0 * 1.2f, wn = s.fw1 * 1.2f;
        float s1 = 1.0f - smooth(0.0f, 0.04f + wl, 0.5f - fabsf(fractf(lat) - 0.5f));
        float s2 = (1.0f - smooth(0.0f, 0.03f + wn, 0.5f - fabsf(fractf(lon) - 0.5f))) *
                   (fabsf(o.z) <= 0.92f ? 1.0f : 0.0f);
        float m = fmaxf(s1, s2);
        a = scale(a, 1.0f - 0.7f * m);
        spec *= 1.0f - 0.8f * m;
    }
    if (rim > 0.5f) {
        const F3 ob = s.obj;
        float wear = 0.6f * noise2(ob.x * 30.0f + ob.z * 17.0f, ob.y * 30.0f + ob.z * 17.0f) +
                     0.4f * noise2(ob.y * 90.0f + ob.x * 41.0f, ob.z * 90.0f + ob.x * 41.0f);
        a = scale(a, mixf(0.7f, 1.15f, wear));
        spec *= mixf(0.4f, 1.4f, wear);
    }
    const F3 sky = ld3(c_sky), gnd = ld3(c_gnd);
    const float hemi = 0.5f + 0.5f * n.z;
    F3 c = vmul(a, F3{mixf(gnd.x, sky.x, hemi), mixf(gnd.y, sky.y, hemi), mixf(gnd.z, sky.z, hemi)});
    float qx = (s.p.x - fr.focus[0]) / 6.0f, qy = (s.p.y - fr.focus[1]) / 6.0f;
    float pool = 0.65f + 0.35f * __expf(-(qx * qx + qy * qy));
    c = c + scale(shade_light(a, spec, gloss, n, v, ld3(fr.sun), ld3(c_sun_col)), lit_k * pool);
    c = c + shade_light(a, spec, gloss, n, v, ld3(fr.fill), ld3(c_fill_col));
    for (int i = 0; i < kLamps; ++i) {
        F3 l = ld3(fr.lamps[i]) - s.p;
        float d2 = dot(l, l);
        if (d2 > 64.0f)
            continue;
        l = scale(l, rsqrtf(d2));
        c = c + scale(shade_light(a, spec, gloss, n, v, l, ld3(c_lamp_col)),
                      smooth(0.25f, 0.8f, l.z) / (1.0f + 0.12f * d2));
    }
    {
        F3 l = ld3(fr.eye_pos) - s.p;
        float d2 = dot(l, l);
        l = scale(l, rsqrtf(d2));
        float cone = smooth(0.35f, 0.85f, -dot(l, ld3(fr.eye_dir)));
        c = c + scale(shade_light(a, spec, gloss, n, v, l, ld3(fr.eye_col)), cone / (1.0f + 2.0f * d2));
    }
    {
        F3 l = ld3(fr.beacon_pos) - s.p;
        float d2 = dot(l, l);
        c = c + scale(shade_light(a, spec, gloss, n, v, scale(l, rsqrtf(d2)), ld3(fr.beacon_col)),
                      1.0f / (1.0f + 1.5f * d2));
    }
    float nv = 1.0f - fmaxf(dot(n, v), 0.0f);
    F3 r = scale(n, 2.0f * dot(n, v)) - v;  // reflect(-v, n)
    float hr = 0.5f + 0.5f * r.z;
    float nv2 = nv * nv, nv4 = nv2 * nv2;
    float sh = spec * (0.04f + 0.5f * nv4 * nv);
    c = c + F3{sh * mixf(gnd.x, 3.0f * sky.x, hr), sh * mixf(gnd.y, 3.0f * sky.y, hr),
               sh * mixf(gnd.z, 3.0f * sky.z, hr)};
    c = c + scale(sky, rim * nv4 * 0.6f);
    if (s.emis >= 0.5f)
        c = scale(a, s.emis);
    c = scale(c, __expf(-kFogDensity * fmaxf(len(ld3(fr.eye) - s.p) - fr.fog_start, 0.0f)));
    c = scale(c, smooth(fr.floor_z - 3.0f, fr.floor_z + 0.2f, s.p.z));
    // ACES fit, then gamma
    float cc[3] = {c.x, c.y, c.z};
    for (int k = 0; k < 3; ++k) {
        float x = cc[k];
        x = x * (2.51f * x + 0.03f) / (x * (2.43f * x + 0.59f) + 0.14f);
        cc[k] = pow_approx(clampf(x, 0.0f, 1.0f), 1.0f / 2.2f);
    }
    return F3{cc[0], cc[1], cc[2]};
}

__device__ __forceinline__ int unorm8(float x) { return (int)floorf(clampf(x, 0.0f, 1.0f) * 255.0f + 0.5f); }

// Additive glow along the ray up to depth tdepth (csrc/arc_render.c:280-302,
// 625-672): halos around glowing parts and beacons, and the beacons' beams.
// `mask`: the billboards that can cover the tile.
__device__ F3 glow_along(const FrameK& fr, unsigned mask, F3 O, F3 D, float tdepth)
{
    F3 g{0.0f, 0.0f, 0.0f};
    const F3 fwd = ld3(fr.fwd), right = ld3(fr.right), up = ld3(fr.up), eye = ld3(fr.eye);
    for (; mask; mask &= mask - 1u) {
        const GlowK& k = fr.glow[__ffs(mask) - 1];
        const F3 c = ld3(k.c);
        float t, u, vv, w;
        if (!k.beam) {
            float den = dot(D, fwd);
            if (den <= 1e-6f)
                continue;
            t = dot(c - O, fwd) / den;
            if (t <= 0.0f || t >= tdepth)
                continue;
            F3 P = O + scale(D, t) - c;
            u = dot(P, right) / k.s;
            vv = dot(P, up) / k.s;
            if (fabsf(u) > 1.0f || fabsf(vv) > 1.0f)
                continue;
            float r2 = u * u + vv * vv;
            float halo = __expf(-6.0f * r2) * 0.8f + __expf(-30.0f * r2);
            w = halo * (1.0f - smooth(0.7f, 1.0f, r2));
        } else {
            const F3 side = ld3(k.side);
            const F3 nb = cross(side, F3{0.0f, 0.0f, 1.0f});
            float den = dot(D, nb);
            if (fabsf(den) <= 1e-9f)
                continue;
            t = dot(c - O, nb) / den;
            if (t <= 0.0f || t >= tdepth)
                continue;
            F3 P = O + scale(D, t) - c;
            u = dot(P, side) / k.s;
            vv = P.z / 3.5f;
            if (fabsf(u) > 1.0f || vv < 0.0f || vv > 1.0f)
                continue;
            w = __expf(-12.0f * u * u) * (1.0f - vv) * (1.0f - vv);
        }
        F3 P = O + scale(D, t);
        w *= k.alpha * __expf(-kFogDensity * fmaxf(len(eye - P) - fr.fog_start, 0.0f));
        g = g + scale(ld3(k.col), w);
    }
    return g;
}

// One CTA per 16 x 16 tile of one world's frame (blockIdx.y: the world).
template <class R>
__global__ void __launch_bounds__(kThreads, ARC_RENDER_MIN_BLOCKS)
    k_render(const VisK* __restrict__ vis, int nv, const FrameK* __restrict__ frames, Worlds<R> W,
             const int* __restrict__ ids, int width, int height, int tiles_x, int samples,
             unsigned char* __restrict__ out)
{
    __shared__ FrameK fr;
    __shared__ unsigned char list[kMaxItems];
    __shared__ int warp_n[kThreads / 32];
    __shared__ unsigned glow_mask;
    const int tid = threadIdx.x, item = blockIdx.y;
    {
        const int* src = reinterpret_cast<const int*>(frames + item);
        int* dst = reinterpret_cast<int*>(&fr);
        for (int i = tid; i < (int)(sizeof(FrameK) / 4); i += kThreads)
            dst[i] = src[i];
    }
    __syncthreads();
    const int world = ids ? ids[item] : item;
    const int tile_x = blockIdx.x % tiles_x, tile_y = blockIdx.x / tiles_x;
    const int x0 = tile_x * kTileW, r0 = tile_y * kTileH;
    const F3 eye = ld3(fr.eye), fwd = ld3(fr.fwd), right = ld3(fr.right), up = ld3(fr.up);
    const float sx = 2.0f / width * fr.tan_y * fr.aspect, sy = 2.0f / height * fr.tan_y;
    // unnormalised ray through window point (wx, wy), y up
    auto ray = [&](float wx, float wy) {
        return fwd + scale(right, (wx - 0.5f * width) * sx) + scale(up, (wy - 0.5f * height) * sy);
    };

    // cull the items' bounding spheres against the tile's frustum
    {
        const float wx0 = (float)x0, wx1 = (float)(x0 + kTileW);
        const float wy1 = (float)(height - r0), wy0 = (float)(height - r0 - kTileH);
        const F3 c00 = ray(wx0, wy0), c10 = ray(wx1, wy0), c11 = ray(wx1, wy1), c01 = ray(wx0, wy1);
        const F3 cc = ray(0.5f * (wx0 + wx1), 0.5f * (wy0 + wy1));
        F3 pn[4] = {cross(c00, c10), cross(c10, c11), cross(c11, c01), cross(c01, c00)};
        for (int k = 0; k < 4; ++k) {
            pn[k] = normalize(pn[k]);
            if (dot(pn[k], cc) > 0.0f)
                pn[k] = -pn[k];
        }
        const int n_items = nv + fr.n_items;
        bool keep = false;
        if (tid < n_items) {
            const VisK& v = tid < nv ? vis[tid] : fr.extra[tid - nv];
            if (v.type >= 0) {
                F3 cw = rot_mul(fr.rot[v.body], ld3(v.bc)) + ld3(fr.pos[v.body]) - eye;
                keep = true;
                for (int k = 0; k < 4; ++k)
                    keep = keep && dot(pn[k], cw) <= v.br;
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if ((tid & 31) == 0)
            warp_n[tid >> 5] = __popc(m);
        __syncthreads();
        int base = 0;
        for (int w = 0; w < (tid >> 5); ++w)
            base += warp_n[w];
        if (keep)
            list[base + __popc(m & ((1u << (tid & 31)) - 1u))] = (unsigned char)tid;
        // the glow billboards' bounding spheres: a halo's square, a beam's quad
        if (tid < 32) {
            bool g = false;
            if (tid < fr.n_glow) {
                const GlowK& k = fr.glow[tid];
                F3 c = ld3(k.c) - eye;
                float rad = 1.4143f * k.s;
                if (k.beam) {
                    c.z += 1.75f;
                    rad = sqrtf(1.75f * 1.75f + k.s * k.s);
                }
                g = true;
                for (int q = 0; q < 4; ++q)
                    g = g && dot(pn[q], c) <= rad;
            }
            const unsigned gm = __ballot_sync(0xffffffffu, g);
            if (tid == 0)
                glow_mask = gm;
        }
    }
    __syncthreads();
    int n_list = 0;
    for (int w = 0; w < kThreads / 32; ++w)
        n_list += warp_n[w];

    TerrainF<R> T;
    T.h = W.th + W.toff[world];
    T.nx = fr.nx;
    T.ny = fr.ny;
    T.cell = fr.cell;
    T.ox = fr.ox;
    T.oy = fr.oy;
    T.outside = fr.outside;
    T.hmax = fr.hmax;
    T.bottom = fr.bottom;

    // each warp takes an 8 x 4 block of the tile: nearby pixels tend to hit
    // the same surfaces, so fewer lanes diverge than along a 32-pixel row
    static_assert(kTileW == 16 && kTileH == 16, "warp blocks laid out for 16 x 16 tiles");
    const int px = x0 + ((tid >> 5) & 1) * 8 + (tid & 7), row = r0 + (tid >> 6) * 4 + ((tid >> 3) & 3);
    if (px >= width || row >= height)
        return;
    const float wy_pix = (float)(height - 1 - row);
    // 4x multisampling positions within the pixel (x right, y up)
    const float spos[4][2] = {{0.375f, 0.125f}, {0.875f, 0.375f}, {0.125f, 0.625f}, {0.625f, 0.875f}};
    float vx = (px + 0.5f) / width - 0.5f, vy = (wy_pix + 0.5f) / height - 0.5f;
    vx *= (float)width / (float)height;
    const float vig = 1.0f - 0.4f * smooth(0.45f, 1.1f, sqrtf(vx * vx + vy * vy));
    const float dither = (hash2(fmaf(fr.time, 61.0f, px + 0.5f), fmaf(fr.time, 61.0f, wy_pix + 0.5f)) - 0.5f) / 255.0f;
    const F3 dDx = scale(right, sx), dDy = scale(up, sy);
    int acc[3] = {0, 0, 0};
    // the surfaces this pixel's samples hit so far and their colours
    int gid0 = -1, gid1 = -1, gid2 = -1, gid3 = -1;
    unsigned gc0 = 0u, gc1 = 0u, gc2 = 0u, gc3 = 0u;
    for (int si = 0; si < samples; ++si) {
        const float wx = samples == 1 ? px + 0.5f : px + spos[si][0];
        const float wy = samples == 1 ? wy_pix + 0.5f : wy_pix + spos[si][1];
        const F3 Du = ray(wx, wy);
        const float inv_len = rsqrtf(dot(Du, Du));
        const F3 D = scale(Du, inv_len);
        float best = kFar / dot(D, fwd);  // the far plane
        int kind = -1, face = 0, cx = 0, cy = 0, sgn = 0, hit_item = -1;
        F3 nl{0, 0, 1};
        float tt = trace_terrain(T, eye, D, best, face, cx, cy, sgn);
        if (tt >= 0.0f) {
            best = tt;
            kind = 0;
        }
        int last_body = -1;
        F3 ol{0, 0, 0}, dl{0, 0, 0};
        for (int li = 0; li < n_list; ++li) {
            const int it = list[li];
            const VisK& v = it < nv ? vis[it] : fr.extra[it - nv];
            if (v.body != last_body) {
                last_body = v.body;
                ol = rot_tmul(fr.rot[v.body], eye - ld3(fr.pos[v.body]));
                dl = rot_tmul(fr.rot[v.body], D);
            }
            {
                // the ray against the visual's bounding sphere first
                const F3 oc = ol - ld3(v.bc);
                const float b = dot(oc, dl), c = dot(oc, oc) - v.br * v.br;
                if (b * b < c || (b > 0.0f && c > 0.0f))
                    continue;
            }
            float t;
            F3 n;
            if (hit_visual(v, ol, dl, best, t, n)) {
                best = t;
                kind = 1;
                hit_item = it;
                nl = n;
            }
        }
        // Multisampling shades once per pixel and primitive: a sample that
        // hits the surface an earlier sample of this pixel hit (the same
        // visual, or the same face of the same column) takes its colour.
        int sid = -1;
        if (kind == 0)
            sid = 1024 + ((cy * kGridMax + cx) << 3) + (face == kFaceTop ? 0 : (face == kFaceX ? 2 : 4) + (sgn > 0));
        else if (kind == 1)
            sid = hit_item;
        unsigned packed = 0u;
        bool fresh = false;
        if (sid >= 0) {
            if (sid == gid0)
                packed = gc0;
            else if (sid == gid1)
                packed = gc1;
            else if (sid == gid2)
                packed = gc2;
            else if (sid == gid3)
                packed = gc3;
            else
                fresh = true;
        }
        if (fresh) {
            Surface s;
            s.p = eye + scale(D, best);
            s.pat = 0;
            s.fw0 = s.fw1 = 0.0f;
            s.g = F3{0, 0, 0};
            s.obj = F3{0, 0, 0};
            if (kind == 0) {
                // csrc/arc_mesh.c:176-255: vertex colours of the column
                const float h = T.at(cx, cy);
                const float x0c = T.ox + cx * T.cell, y0c = T.oy + cy * T.cell;
                float cb = 0.36f + 0.05f * (float)cell_hash(cx, cy) + 0.09f * clampf(h, -0.3f, 0.4f);
                F3 col;
                if (face == kFaceTop) {
                    s.n = F3{0.0f, 0.0f, 1.0f};
                    auto occ = [&](int ix, int iy) { return clampf((T.at(ix, iy) - h) / 0.12f, 0.0f, 1.0f); };
                    auto corner = [&](int qx, int qy) {
                        float o = occ(cx + qx, cy) + occ(cx, cy + qy) + 0.5f * occ(cx + qx, cy + qy);
                        return cb * (1.0f - 0.22f * o);
                    };
                    const float k00 = corner(-1, -1), k10 = corner(1, -1), k11 = corner(1, 1), k01 = corner(-1, 1);
                    const float u = clampf((s.p.x - x0c) / T.cell, 0.0f, 1.0f);
                    const float w = clampf((s.p.y - y0c) / T.cell, 0.0f, 1.0f);
                    // triangles (00, 10, 11) and (00, 11, 01)
                    const float k = u >= w ? k00 + u * (k10 - k00) + w * (k11 - k10)
                                           : k00 + w * (k01 - k00) + u * (k11 - k01);
                    col = F3{k, k, 1.04f * k};
                } else {
                    const float cs = 0.8f * cb;
                    int nx_ = cx, ny_ = cy;
                    if (face == kFaceX) {
                        nx_ -= sgn;
                        s.n = F3{(float)-sgn, 0.0f, 0.0f};
                    } else {
                        ny_ -= sgn;
                        s.n = F3{0.0f, (float)-sgn, 0.0f};
                    }
                    const float zlo = fmaxf(T.at(nx_, ny_), T.bottom);
                    const float f = h > zlo ? clampf((s.p.z - zlo) / (h - zlo), 0.0f, 1.0f) : 1.0f;
                    col = F3{mixf(0.45f * cs, cs, f), mixf(0.45f * cs, cs, f), mixf(0.47f * cs, 1.04f * cs, f)};
                }
                s.albedo = vmul(col, col);
                s.spec = 0.25f;
                s.gloss = 16.0f;
                s.emis = 0.0f;
                s.rim = 0.0f;
                s.pat = 1;
                s.g = F3{(s.p.x - T.ox) / T.cell, (s.p.y - T.oy) / T.cell, 0.0f};
                // fwidth(g.x) + fwidth(g.y) from the neighbouring pixels' rays on this plane
                float w = 0.0f;
                const float pn = dot(s.p - eye, s.n);
                for (int k = 0; k < 2; ++k) {
                    F3 D2 = Du + (k ? dDy : dDx);
                    float den = dot(D2, s.n);
                    F3 dp = fabsf(den) > 1e-9f ? eye + scale(D2, pn / den) - s.p : F3{1e3f, 1e3f, 1e3f};
                    w += (fabsf(dp.x) + fabsf(dp.y)) / T.cell;
                }
                s.fw0 = w;
            } else {
                const VisK& v = hit_item < nv ? vis[hit_item] : fr.extra[hit_item - nv];
                const float* rm = fr.rot[v.body];
                s.n = normalize(rot_mul(rm, nl));
                const F3 col = ld3(v.col);
                s.albedo = vmul(col, col);
                const int m = v.material >= 0 && v.material <= kMatGlow ? v.material : 0;
                s.spec = c_mat[m][0];
                s.gloss = c_mat[m][1];
                s.emis = c_mat[m][2];
                s.pat = (int)c_mat[m][3];
                s.rim = v.rim;
                const F3 pl = rot_tmul(rm, s.p - ld3(fr.pos[v.body]));  // body frame
                s.obj = v.type == kVisSphere ? scale(pl - ld3(v.o), 1.0f / v.a) : pl;
                if (s.pat == 2) {
                    const F3 o = normalize(s.obj);
                    s.g = o;
                    const float pn = dot(s.p - eye, s.n);
                    float wl = 0.0f, wn = 0.0f;
                    const float ct = sqrtf(fmaxf(1.0f - o.z * o.z, 1e-12f)), rxy = fmaxf(o.x * o.x + o.y * o.y, 1e-12f);
                    for (int k = 0; k < 2; ++k) {
                        F3 D2 = Du + (k ? dDy : dDx);
                        float den = dot(D2, s.n);
                        F3 dp = fabsf(den) > 1e-9f ? eye + scale(D2, pn / den) - s.p : F3{1e3f, 1e3f, 1e3f};
                        F3 dob = scale(rot_tmul(rm, dp), 1.0f / v.a);
                        wl += fabsf(dob.z / ct) * 7.0f / 3.14159f;
                        wn += fabsf((o.x * dob.y - o.y * dob.x) / rxy) * 6.0f / 3.14159f;
                    }
                    s.fw0 = wl;
                    s.fw1 = wn;
                }
            }
            // key light visibility: the shadow map's region fades out at its edge
            const F3 pb = s.p + scale(s.n, kShadowNormalOffset);
            float ex = fabsf(dot(pb, ld3(fr.sl)) - fr.shadow_c[0]) / (float)(2.0 * kShadowRange);
            float ey = fabsf(dot(pb, ld3(fr.ul)) - fr.shadow_c[1]) / (float)(2.0 * kShadowRange);
            const float fade = smooth(0.5f, 0.42f, fmaxf(ex, ey));
            float lit_k = 1.0f;
            if (fade > 0.0f && dot(s.n, ld3(fr.sun)) > 0.0f) {
                const float k = shadowed(fr, T, vis, nv, s.p + scale(s.n, 2e-3f)) ? 0.0f : 1.0f;
                lit_k = mixf(1.0f, k, fade);
            }
            const F3 c = shade_scene(fr, s, lit_k);
            packed = (unsigned)unorm8(c.x + dither) | (unsigned)unorm8(c.y + dither) << 8 |
                     (unsigned)unorm8(c.z + dither) << 16;
            if (gid0 < 0) {
                gid0 = sid;
                gc0 = packed;
            } else if (gid1 < 0) {
                gid1 = sid;
                gc1 = packed;
            } else if (gid2 < 0) {
                gid2 = sid;
                gc2 = packed;
            } else {
                gid3 = sid;
                gc3 = packed;
            }
        }
        const int s8[3] = {(int)(packed & 255u), (int)((packed >> 8) & 255u), (int)(packed >> 16)};
        // additive glow (depth tested, not written), then the vignette
        const F3 g = glow_along(fr, glow_mask, eye, D, kind >= 0 ? best : 1e30f);
        const float gg[3] = {g.x, g.y, g.z};
        for (int k = 0; k < 3; ++k) {
            int v8 = unorm8(s8[k] / 255.0f + gg[k]);
            acc[k] += (int)floorf(v8 * vig + 0.5f);
        }
    }
    unsigned char* o = out + (((size_t)item * height + row) * width + px) * 3;
    for (int k = 0; k < 3; ++k)
        o[k] = (unsigned char)((acc[k] + samples / 2) / samples);
}

__device__ __forceinline__ double wrap_angle(double a)
{
    for (int i = 0; i < 64 && a > kPi; ++i)
        a -= 2.0 * kPi;
    for (int i = 0; i < 64 && a < -kPi; ++i)
        a += 2.0 * kPi;
    return a;
}

// Height of the column containing (x, y) (csrc/arc_terrain.h:42-50), with
// the terrain's FP64 geometry, as the reference computes it.
template <class R> __device__ double height_at(const TerrainGeomD& g, const R* h, double x, double y)
{
    double fx = floor((x - g.ox) / g.cell), fy = floor((y - g.oy) / g.cell);
    if (!(fx >= 0.0 && fy >= 0.0 && fx < g.nx && fy < g.ny))
        return g.outside;
    return (double)h[(int)fx + (int)fy * g.nx];
}

__device__ __forceinline__ void put3(float* d, double x, double y, double z)
{
    d[0] = (float)x;
    d[1] = (float)y;
    d[2] = (float)z;
}

__device__ __forceinline__ double warp_min(double v)
{
    for (int o = 16; o > 0; o >>= 1)
        v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_max(double v)
{
    for (int o = 16; o > 0; o >>= 1)
        v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

constexpr int kSetupWarps = 2;  // rendered worlds per CTA of k_frame_setup

// One warp per rendered world: the lanes split the terrain's lowest and
// highest column, the lamps' heights, the body poses, the visuals' bounding
// spheres and glow billboards; lane 0 then writes the camera, lights and
// markers.
template <class R>
__global__ void __launch_bounds__(32 * kSetupWarps)
    k_frame_setup(Worlds<R> W, const VisK* __restrict__ vis, int nv, int eye_vis, const int* __restrict__ ids,
                  int n, const float* __restrict__ markers, int mpw, const int* __restrict__ active,
                  CamState* __restrict__ cams, int cam_slot, CamParams cp, FrameK* __restrict__ frames)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x / 32;
    const int item = blockIdx.x * kSetupWarps + warp;
    __shared__ float s_body_r[kSetupWarps][kPoses];
    if (item >= n)
        return;  // the whole warp
    const int world = ids ? ids[item] : item;
    FrameK& f = frames[item];
    const R* rec = W.rec + (size_t)world * W.stride;
    const int nb = W.off_sphere / kBodyRec;
    auto body_x = [&](int b) {
        const R* p = rec + b * kBodyRec;
        return V3<double>{(double)p[0], (double)p[1], (double)p[2]};
    };
    auto body_q = [&](int b) {
        const R* p = rec + b * kBodyRec;
        return Q4<double>{(double)p[3], (double)p[4], (double)p[5], (double)p[6]};
    };
    // terrain: lowest and highest column, lamps (csrc/arc_render.c:523-549)
    const TerrainView<R> tv = terrain_of(W, world);
    double lo = 1e30, hi = -1e30;
    for (int k = lane; k < tv.nx * tv.ny; k += 32) {
        double h = (double)tv.h[k];
        lo = fmin(lo, h);
        hi = fmax(hi, h);
    }
    lo = warp_min(lo);
    hi = warp_max(hi);
    if (tv.nx * tv.ny == 0)
        lo = hi = 0.0;
    // Each lamp takes the highest column among samples at offsets that
    // accumulate in steps of half a cell from -1 m to 1 m, as the reference's
    // loops do. The lanes split the (lamp, x offset) pairs; a lane rebuilds
    // its x offset by the same accumulation.
    const TerrainGeomD gd = W.tgd[world];
    const double step = 0.5 * gd.cell;
    int count = 0;
    for (double d = -1.0; d <= 1.0 && count < (1 << 16); d += step)
        ++count;
    auto lamp_x = [&](int k) { return gd.ox + gd.nx * gd.cell * (k % kLampGrid + 0.5) / kLampGrid; };
    auto lamp_y = [&](int k) { return gd.oy + gd.ny * gd.cell * (k / kLampGrid + 0.5) / kLampGrid; };
    double tops[kLamps];
#pragma unroll
    for (int k = 0; k < kLamps; ++k)
        tops[k] = lo;
    for (int q = lane; q < kLamps * count; q += 32) {
        const int k = q / count, i = q % count;
        double dx = -1.0;
        for (int a = 0; a < i; ++a)
            dx += step;
        const double x = lamp_x(k) + dx, y = lamp_y(k);
        double top = lo;
        int guard = 0;
        for (double dy = -1.0; dy <= 1.0 && guard < (1 << 16); dy += step, ++guard)
            top = fmax(top, height_at(gd, tv.h, x, y + dy));
#pragma unroll
        for (int kk = 0; kk < kLamps; ++kk)
            if (kk == k)
                tops[kk] = fmax(tops[kk], top);
    }
#pragma unroll
    for (int k = 0; k < kLamps; ++k) {
        const double top = warp_max(tops[k]);
        if (lane == 0)
            put3(f.lamps[k], lamp_x(k), lamp_y(k), top + kLampHeight);
    }
    // body poses (csrc/arc_render.c:453-469), one lane per body
    if (lane < kPoses) {
        const int b = lane;
        double x[3] = {0, 0, 0}, m[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
        if (b < nb && b < kMaxBodies) {
            const V3<double> bxx = body_x(b);
            const Q4<double> q = body_q(b);
            x[0] = bxx.x;
            x[1] = bxx.y;
            x[2] = bxx.z;
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
        put3(f.pos[b], x[0], x[1], x[2]);
        for (int k = 0; k < 9; ++k)
            f.rot[b][k] = (float)m[k];
        s_body_r[warp][b] = 0.0f;
    }
    // camera (csrc/arc_render.c:700-716, 1040-1062): every lane computes it,
    // lane 0 stores the smoothing state
    CamState& cs = cams[cam_slot >= 0 ? cam_slot : world];
    const V3<double> x0 = body_x(0);
    const Q4<double> q0 = body_q(0);
    const V3<double> fwd_body = qrotate(q0, V3<double>{1, 0, 0});
    const double heading = atan2(fwd_body.y, fwd_body.x);
    const V3<double> target = x0 + V3<double>{0, 0, 0.1};
    V3<double> ct{cs.target[0], cs.target[1], cs.target[2]};
    double cam_heading = cs.heading;
    __syncwarp();
    if (!cs.init || len(target - ct) > 3.0) {
        ct = target;
        cam_heading = heading;
    }
    ct = ct + scale(target - ct, 0.15);
    cam_heading += 0.03 * wrap_angle(heading - cam_heading);
    __syncwarp();
    if (lane == 0) {
        cs.init = 1;
        cs.heading = cam_heading;
        cs.target[0] = ct.x;
        cs.target[1] = ct.y;
        cs.target[2] = ct.z;
    }
    const double yaw = cam_heading + kPi + cp.yaw;
    V3<double> eye = ct + V3<double>{cp.dist * cos(cp.pitch) * cos(yaw), cp.dist * cos(cp.pitch) * sin(yaw),
                                     cp.dist * sin(cp.pitch)};
    eye.z = fmax(eye.z, height_at(gd, tv.h, eye.x, eye.y) + 0.2);
    // bounding spheres of the shadow casters (the robot's, and each body's,
    // centred on the body) and the robot's glow billboards, in visual order
    // (csrc/arc_render.c:636-646), the lanes splitting the visuals
    double rr = 0.0;
    int ng = 0;
    for (int base = 0; base < nv; base += 32) {
        const int i = base + lane;
        bool glow = false;
        V3<double> c{0, 0, 0};
        double sz = 0.0;
        if (i < nv && vis[i].type >= 0) {
            const VisK& v = vis[i];
            const V3<double> bxx = body_x(v.body);
            const Q4<double> bqq = body_q(v.body);
            if (!v.glow) {
                const V3<double> cw = bxx + qrotate(bqq, V3<double>{v.bc[0], v.bc[1], v.bc[2]});
                rr = fmax(rr, len(cw - x0) + v.br);
                atomicMax(reinterpret_cast<int*>(&s_body_r[warp][v.body]),
                          __float_as_int((float)(len(cw - bxx) + v.br)));
            } else {
                V3<double> local = v.type == kVisCylinder
                                       ? V3<double>{v.o[0] + 0.5 * v.b * v.d[0], v.o[1] + 0.5 * v.b * v.d[1],
                                                    v.o[2] + 0.5 * v.b * v.d[2]}
                                       : V3<double>{v.o[0], v.o[1], v.o[2]};
                if (v.type == kVisTaper)
                    local = V3<double>{v.bc[0], v.bc[1], v.bc[2]};
                c = bxx + qrotate(bqq, local);
                sz = v.type == kVisRing ? 1.7 * (v.a + v.b) : 3.5 * v.a;
                glow = true;
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, glow);
        const int pos = ng + __popc(m & ((1u << lane) - 1u));
        if (glow && pos < kMaxGlow) {
            const VisK& v = vis[i];
            const V3<double> bc = c + scale(normalize(eye - c), 0.6 * sz);
            GlowK& g = f.glow[pos];
            put3(g.c, bc.x, bc.y, bc.z);
            g.s = (float)sz;
            put3(g.col, v.col[0], v.col[1], v.col[2]);
            g.alpha = v.type == kVisRing ? 0.4f : 0.3f;
            g.beam = 0;
        }
        ng = min(ng + __popc(m), kMaxGlow);
    }
    rr = warp_max(rr);
    __syncwarp();
    if (lane < kPoses) {
        const int b = lane;
        const float r = s_body_r[warp][b];
        const bool has = b < nb && b < kMaxBodies && r > 0.0f;
        const V3<double> bxx = has ? body_x(b) : V3<double>{0, 0, 0};
        put3(f.body_c[b], bxx.x, bxx.y, bxx.z);
        f.body_r[b] = has ? r + 1e-3f : 0.0f;
    }
    if (lane != 0)
        return;
    const V3<double> bx0 = x0;
    const Q4<double> bq0 = q0;
    f.nx = tv.nx;
    f.ny = tv.ny;
    f.cell = (float)tv.cell;
    f.ox = (float)tv.ox;
    f.oy = (float)tv.oy;
    f.outside = (float)tv.outside;
    f.floor_z = (float)lo;
    f.bottom = (float)(lo - kVoidDepth);
    f.hmax = (float)hi;
    const V3<double> fz = normalize(ct - eye);
    const V3<double> sx = normalize(cross(fz, V3<double>{0, 0, 1}));
    const V3<double> uy = cross(sx, fz);
    put3(f.eye, eye.x, eye.y, eye.z);
    put3(f.fwd, fz.x, fz.y, fz.z);
    put3(f.right, sx.x, sx.y, sx.z);
    put3(f.up, uy.x, uy.y, uy.z);
    f.tan_y = (float)tan(0.5 * 50.0 * kPi / 180.0);
    f.aspect = (float)((double)cp.width / (cp.height > 0 ? cp.height : 1));
    f.fog_start = (float)len(eye - ct);
    const double time = W.time[world];
    f.time = (float)time - floorf((float)time);
    f.focus[0] = (float)ct.x;
    f.focus[1] = (float)ct.y;
    // lights
    const V3<double> sun = normalize(V3<double>{kSunDir[0], kSunDir[1], kSunDir[2]});
    const V3<double> fill = normalize(V3<double>{kFillDir[0], kFillDir[1], kFillDir[2]});
    put3(f.sun, sun.x, sun.y, sun.z);
    put3(f.fill, fill.x, fill.y, fill.z);
    {
        // light space of the shadow map, its square snapped to whole texels (csrc/arc_render.c:986-998)
        const V3<double> lf = -sun;
        const V3<double> ls = normalize(cross(lf, V3<double>{0, 0, 1}));
        const V3<double> lu = cross(ls, lf);
        put3(f.sl, ls.x, ls.y, ls.z);
        put3(f.ul, lu.x, lu.y, lu.z);
        f.shadow_c[0] = (float)(floor(dot(ls, ct) / kShadowTexel) * kShadowTexel);
        f.shadow_c[1] = (float)(floor(dot(lu, ct) / kShadowTexel) * kShadowTexel);
    }
    put3(f.eye_pos, 0, 0, -100);
    put3(f.eye_dir, 1, 0, 0);
    put3(f.eye_col, 0, 0, 0);
    if (eye_vis >= 0) {  // csrc/arc_render.c:1010-1023
        const VisK& v = vis[eye_vis];
        const float* ax = v.d;
        const V3<double> axis = qrotate(bq0, normalize(V3<double>{ax[0], ax[1], ax[2]}));
        const V3<double> c = bx0 + qrotate(bq0, V3<double>{v.o[0], v.o[1], v.o[2]});
        const V3<double> ep = c + scale(axis, 0.05);
        const V3<double> ed = normalize(axis + V3<double>{0, 0, -0.35});
        put3(f.eye_pos, ep.x, ep.y, ep.z);
        put3(f.eye_dir, ed.x, ed.y, ed.z);
        put3(f.eye_col, kEyeLight * v.col[0] * v.col[0], kEyeLight * v.col[1] * v.col[1],
             kEyeLight * v.col[2] * v.col[2]);
    }
    const int act = active ? active[item] : -1;
    const int nm = markers ? mpw : 0;
    const float* mk = markers ? markers + (size_t)item * mpw * 4 : nullptr;
    put3(f.beacon_pos, 0, 0, -100);
    put3(f.beacon_col, 0, 0, 0);
    if (nm > 0) {
        const float* c = act == 0 ? c_beacon_seen : c_beacon_unseen;
        const double k = act == 0 ? 1.6 : 0.8;
        put3(f.beacon_pos, mk[0], mk[1], (double)mk[2] + kBeaconHeight);
        put3(f.beacon_col, k * c[0], k * c[1], k * c[2]);
    }
    f.robot_c[0] = (float)bx0.x;
    f.robot_c[1] = (float)bx0.y;
    f.robot_c[2] = (float)bx0.z;
    f.robot_r = (float)rr + 1e-3f;
    // markers: beacon spheres and rings (emissive), halos and beams (csrc/arc_render.c:566-599, 647-671)
    int ne = 0;
    for (int i = 0; i < nm && i < kMaxMarkers; ++i) {
        const float* m = mk + 4 * i;
        const float* c = i == act ? c_beacon_seen : c_beacon_unseen;
        const V3<double> p{m[0], m[1], (double)m[2] + kBeaconHeight + 0.06 * sin(3.0 * time)};
        for (int e = 0; e < 2; ++e) {
            VisK& v = f.extra[ne++];
            v.type = e == 0 ? kVisSphere : kVisRing;
            v.body = kIdentity;
            v.material = kMatGlow;
            v.glow = 1;
            for (int k = 0; k < 3; ++k)
                v.col[k] = sqrtf(c[k]);
            v.rim = 0.0f;
            if (e == 0) {
                put3(v.o, p.x, p.y, p.z);
                v.a = 0.07f;
                v.br = 0.07f;
            } else {
                put3(v.o, m[0], m[1], (double)m[2] + 0.01);
                put3(v.d, 0, 0, 1);
                v.a = m[3];
                v.b = 0.012f;
                v.br = m[3] + 0.012f;
            }
            for (int k = 0; k < 3; ++k)
                v.bc[k] = v.o[k];
        }
        if (ng + 2 <= kMaxGlow) {
            GlowK& h = f.glow[ng++];
            const V3<double> bc = p + scale(normalize(eye - p), 0.3);
            put3(h.c, bc.x, bc.y, bc.z);
            h.s = 0.45f;
            put3(h.col, c[0], c[1], c[2]);
            h.alpha = 0.8f;
            h.beam = 0;
            GlowK& b = f.glow[ng++];
            const V3<double> base{m[0], m[1], m[2]};
            const V3<double> side = normalize(cross(V3<double>{0, 0, 1}, eye - base));
            put3(b.c, base.x, base.y, base.z);
            put3(b.side, side.x, side.y, side.z);
            b.s = 0.1f;
            put3(b.col, c[0], c[1], c[2]);
            b.alpha = 0.5f;
            b.beam = 1;
        }
    }
    f.n_items = ne;
    f.n_glow = ng;
}

// The checkpoint of each world of a device env as its marker, highlighted
// while the robot sees it (ArcTask.markers and Viewer.render,
// arc/task.py:261-264, arc/env.py:45-47).
__global__ void k_env_markers(TaskState S, double radius, const int* __restrict__ ids, int n,
                              float* __restrict__ markers, int* __restrict__ active)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    const int w = ids ? ids[k] : k;
    markers[4 * k + 0] = (float)S.target[2 * w];
    markers[4 * k + 1] = (float)S.target[2 * w + 1];
    markers[4 * k + 2] = (float)S.target_z[w];
    markers[4 * k + 3] = (float)radius;
    active[k] = S.in_view[w] ? 0 : -1;
}

}  // namespace rd

// ---- host

namespace {

using namespace rd;
using V3d = V3<double>;

void seg_frame(V3d p0, V3d p1, V3d& d, V3d& u, V3d& v, double& L)
{
    V3d s = p1 - p0;
    L = len(s);
    d = scale(s, 1.0 / (L > 1e-12 ? L : 1.0));
    if (fabs(d.x) < 1e-9 && fabs(d.y) < 1e-9) {
        u = V3d{1, 0, 0};
        v = V3d{0, d.z > 0 ? 1.0 : -1.0, 0};
    } else {
        u = normalize(fabs(d.z) < 0.9 ? cross(V3d{0, 0, 1}, d) : cross(V3d{1, 0, 0}, d));
        v = cross(d, u);
    }
}

void put(float* dst, V3d a)
{
    dst[0] = (float)a.x;
    dst[1] = (float)a.y;
    dst[2] = (float)a.z;
}

// The intersection form of a visual (csrc/arc_mesh.c:12-177 define the shapes).
VisK make_vis(const ModelHost::Visual& s)
{
    VisK v;
    std::memset(&v, 0, sizeof(v));
    v.type = s.type;
    v.body = s.body;
    v.material = s.material;
    v.glow = s.material == kMatGlow;
    for (int k = 0; k < 3; ++k)
        v.col[k] = s.color[k];
    v.rim = 1.0f;
    switch (s.type) {
    case kVisSphere:
        put(v.o, s.p0);
        v.a = (float)s.radius;
        put(v.bc, s.p0);
        v.br = (float)s.radius;
        break;
    case kVisBox: {
        const V3d e = s.p1;
        const double bevel = 0.22 * fmin(e.x, fmin(e.y, e.z));
        put(v.o, s.p0);
        v.a = (float)(e.x - bevel);
        v.b = (float)(e.y - bevel);
        v.c = (float)(e.z - bevel);
        v.e = (float)bevel;
        put(v.bc, s.p0);
        v.br = (float)len(e) + 1e-4f;
        break;
    }
    case kVisTaper: {
        static const double PX[8] = {1, 0.6, -0.6, -1, -1, -0.6, 0.6, 1};
        static const double PY[8] = {0.45, 1, 1, 0.45, -0.45, -1, -1, -0.45};
        V3d d, u, w;
        double L;
        seg_frame(s.p0, s.p1, d, u, w, L);
        if (L < 1e-9) {
            v.type = -1;
            break;
        }
        V3d a[8], b[8];
        double cross_r = 0.0;
        for (int k = 0; k < 8; ++k) {
            a[k] = s.p0 + scale(u, PX[k] * s.radius) + scale(w, PY[k] * s.radius * s.aspect);
            b[k] = s.p0 + scale(d, L) + scale(u, PX[k] * s.radius2) + scale(w, PY[k] * s.radius2 * s.aspect);
            cross_r = fmax(cross_r, fmax(len(a[k] - s.p0), len(b[k] - (s.p0 + scale(d, L)))));
        }
        for (int k = 0; k < 8; ++k) {
            const int m = (k + 1) % 8;
            V3d n = normalize(cross(a[m] - a[k], b[k] - a[k]));
            if (dot(n, a[k] - s.p0) < 0.0)
                n = -n;
            put(v.pl[k], n);
            v.pl[k][3] = (float)dot(n, a[k]);
        }
        put(v.pl[8], -d);
        v.pl[8][3] = (float)dot(-d, s.p0);
        put(v.pl[9], d);
        v.pl[9][3] = (float)dot(d, s.p0 + scale(d, L));
        put(v.o, s.p0);
        put(v.d, d);
        v.b = (float)L;
        put(v.bc, s.p0 + scale(d, 0.5 * L));
        v.br = (float)sqrt(0.25 * L * L + cross_r * cross_r) + 1e-4f;
        break;
    }
    case kVisCylinder: {
        V3d d, u, w;
        double L;
        seg_frame(s.p0, s.p1, d, u, w, L);
        if (L < 1e-9) {
            v.type = -1;
            break;
        }
        put(v.o, s.p0);
        put(v.d, d);
        v.a = (float)s.radius;
        v.b = (float)L;
        if (s.material == kMatRibs) {  // csrc/arc_mesh.c:71-72
            v.c = (float)(0.12 * s.radius);
            v.e = (float)(2.0 / 0.010);  // sin(2 pi z / pitch) = sinpi(e z)
        }
        put(v.bc, s.p0 + scale(d, 0.5 * L));
        v.br = (float)sqrt(0.25 * L * L + s.radius * s.radius) + 1e-4f;
        break;
    }
    case kVisRing:
        put(v.o, s.p0);
        put(v.d, normalize(s.p1));
        v.a = (float)s.radius;
        v.b = (float)s.radius2;
        put(v.bc, s.p0);
        v.br = (float)(s.radius + s.radius2) + 1e-4f;
        break;
    default:
        v.type = -1;
    }
    return v;
}

}  // namespace
}  // namespace arc

using namespace arc;

struct arc_renderer {
    int w = 0, h = 0, samples = 4, view = 0;
    double yaw = 0.5, pitch = 0.3, dist = 4.0;
    // visuals of the last model drawn, on the device
    std::vector<ModelHost::Visual> vis_host;
    rd::VisK* d_vis = nullptr;
    int nv = 0, eye_vis = -1;
    // cameras: one per world of `cam_sim`, plus the single-frame camera
    const arc_sim* cam_sim = nullptr;
    int cam_n = 0;
    rd::CamState* d_cams = nullptr;
    rd::FrameK* d_frames = nullptr;
    int frames_cap = 0;
    unsigned char* d_rgb = nullptr;
    float* d_markers = nullptr;
    int* d_ids = nullptr;
    int* d_active = nullptr;
    int markers_cap = 0;
    unsigned char* h_scratch = nullptr;
    // markers of arc_env_render
    float* d_env_markers = nullptr;
    int* d_env_active = nullptr;
    int env_cap = 0;
    cudaEvent_t done = nullptr;  // the last call's kernels
    bool used = false;
};

namespace {

int report(cudaError_t e, const char* where)
{
    if (e == cudaSuccess)
        return ARC_OK;
    std::fprintf(stderr, "arc_render: %s: %s\n", where, cudaGetErrorString(e));
    return ARC_ERR_CUDA;
}

// Uploads the visuals of the sim's model when they differ from the last ones.
int sync_visuals(arc_renderer* r, const SimView& sv)
{
    const ModelHost& m = *sv.model;
    bool same = (int)r->vis_host.size() == m.nv &&
                (m.nv == 0 || !std::memcmp(r->vis_host.data(), m.v, sizeof(ModelHost::Visual) * m.nv));
    if (same && (r->d_vis || m.nv == 0))
        return ARC_OK;
    std::vector<rd::VisK> k(m.nv);
    r->eye_vis = -1;
    for (int i = 0; i < m.nv; ++i) {
        k[i] = make_vis(m.v[i]);
        if (r->eye_vis < 0 && m.v[i].material == kMatGlow && m.v[i].type == kVisRing && m.v[i].body == 0)
            r->eye_vis = i;
    }
    if (r->d_vis)
        cudaFree(r->d_vis);
    r->d_vis = nullptr;
    if (m.nv > 0) {
        if (report(cudaMalloc((void**)&r->d_vis, sizeof(rd::VisK) * m.nv), "cudaMalloc(visuals)"))
            return ARC_ERR_CUDA;
        if (report(cudaMemcpy(r->d_vis, k.data(), sizeof(rd::VisK) * m.nv, cudaMemcpyHostToDevice), "visuals"))
            return ARC_ERR_CUDA;
    }
    r->vis_host.assign(m.v, m.v + m.nv);
    r->nv = m.nv;
    return ARC_OK;
}

// Cameras for every world of s plus one for arc_render_frame (slot n),
// zeroed on the stream of the launch that first reads them (the sim's
// stream does not synchronise with the legacy default stream).
int sync_cameras(arc_renderer* r, const arc_sim* s, int n, cudaStream_t st)
{
    if (r->cam_sim == s && r->cam_n == n && r->d_cams)
        return ARC_OK;
    if (r->d_cams)
        cudaFree(r->d_cams);
    r->d_cams = nullptr;
    if (report(cudaMalloc((void**)&r->d_cams, sizeof(rd::CamState) * (n + 1)), "cudaMalloc(cameras)"))
        return ARC_ERR_CUDA;
    if (report(cudaMemsetAsync(r->d_cams, 0, sizeof(rd::CamState) * (n + 1), st), "cameras"))
        return ARC_ERR_CUDA;
    r->cam_sim = s;
    r->cam_n = n;
    return ARC_OK;
}

int grow_frames(arc_renderer* r, int n)
{
    if (n <= r->frames_cap)
        return ARC_OK;
    if (r->d_frames)
        cudaFree(r->d_frames);
    r->d_frames = nullptr;
    r->frames_cap = 0;
    if (report(cudaMalloc((void**)&r->d_frames, sizeof(rd::FrameK) * n), "cudaMalloc(frames)"))
        return ARC_ERR_CUDA;
    r->frames_cap = n;
    return ARC_OK;
}

template <class R>
int launch(arc_renderer* r, const SimView& sv, const Worlds<R>& W, const int* d_ids, int n, const float* d_markers,
           int mpw, const int* d_active, int cam_slot, unsigned char* d_rgb, cudaStream_t st)
{
    rd::CamParams cp{r->yaw, r->pitch, r->dist, r->w, r->h};
    rd::k_frame_setup<R><<<(n + rd::kSetupWarps - 1) / rd::kSetupWarps, 32 * rd::kSetupWarps, 0, st>>>(W, r->d_vis, r->nv, r->eye_vis, d_ids, n, d_markers, mpw,
                                                       d_active, r->d_cams, cam_slot, cp, r->d_frames);
    if (report(cudaGetLastError(), "frame setup"))
        return ARC_ERR_CUDA;
    const int tiles_x = (r->w + rd::kTileW - 1) / rd::kTileW, tiles_y = (r->h + rd::kTileH - 1) / rd::kTileH;
    dim3 grid(tiles_x * tiles_y, n);
    rd::k_render<R><<<grid, rd::kThreads, 0, st>>>(r->d_vis, r->nv, r->d_frames, W, d_ids, r->w, r->h, tiles_x,
                                                   r->samples, d_rgb);
    return report(cudaGetLastError(), "render");
}

int render_any(arc_renderer* r, const arc_sim* s, const int* d_ids, int n, const float* d_markers, int mpw,
               const int* d_active, int cam_slot, unsigned char* d_rgb, cudaStream_t st)
{
    const SimView sv = sim_view(s);
    int rc;
    // calls share the frame records and cameras: a call on another stream
    // waits for the previous call's kernels
    if (r->used && report(cudaStreamWaitEvent(st, r->done, 0), "stream wait"))
        return ARC_ERR_CUDA;
    if ((rc = sync_visuals(r, sv)) || (rc = sync_cameras(r, s, sv.n, st)) || (rc = grow_frames(r, n)))
        return rc;
    if (r->nv > kMaxVisuals)
        return ARC_ERR_ARG;
    rc = sv.fp64 ? launch<double>(r, sv, sv.wd, d_ids, n, d_markers, mpw, d_active, cam_slot, d_rgb, st)
                 : launch<float>(r, sv, sv.wf, d_ids, n, d_markers, mpw, d_active, cam_slot, d_rgb, st);
    if (rc == ARC_OK) {
        if (report(cudaEventRecord(r->done, st), "event"))
            return ARC_ERR_CUDA;
        r->used = true;
    }
    return rc;
}

}  // namespace

extern "C" {

arc_renderer* arc_render_create(int width, int height, int visible)
{
    if (visible || width <= 0 || height <= 0 || width > 16384 || height > 16384)
        return nullptr;
    arc_renderer* r = new (std::nothrow) arc_renderer();
    if (!r)
        return nullptr;
    r->w = width;
    r->h = height;
    arc_render_set_view(r, 0);
    const size_t bytes = (size_t)width * height * 3;
    if (cudaMalloc((void**)&r->d_rgb, bytes) != cudaSuccess ||
        cudaMalloc((void**)&r->d_markers, sizeof(float) * 4 * rd::kMaxMarkers) != cudaSuccess ||
        cudaMalloc((void**)&r->d_ids, sizeof(int) * 2) != cudaSuccess ||
        cudaMallocHost((void**)&r->h_scratch, bytes) != cudaSuccess ||
        cudaEventCreateWithFlags(&r->done, cudaEventDisableTiming) != cudaSuccess) {
        arc_render_destroy(r);
        return nullptr;
    }
    r->d_active = r->d_ids + 1;
    return r;
}

void arc_render_destroy(arc_renderer* r)
{
    if (!r)
        return;
    cudaFree(r->d_vis);
    cudaFree(r->d_cams);
    cudaFree(r->d_frames);
    cudaFree(r->d_rgb);
    cudaFree(r->d_markers);
    cudaFree(r->d_ids);
    cudaFree(r->d_env_markers);
    cudaFree(r->d_env_active);
    cudaFreeHost(r->h_scratch);
    if (r->done)
        cudaEventDestroy(r->done);
    delete r;
}

int arc_render_frame(arc_renderer* r, const arc_sim* s, int world, const double* markers, int n_markers, int active,
                     unsigned char* rgb)
{
    if (!r || !s)
        return 0;
    if (world < 0 || world >= arc_sim_num_worlds(s)) {
        std::fprintf(stderr, "arc_render: world %d out of range\n", world);
        return 0;
    }
    if (!markers)
        n_markers = 0;
    if (n_markers > rd::kMaxMarkers)
        n_markers = rd::kMaxMarkers;
    cudaStream_t st = (cudaStream_t)arc_sim_stream(s);
    float m[4 * rd::kMaxMarkers] = {};
    for (int i = 0; i < 4 * n_markers; ++i)
        m[i] = (float)markers[i];
    int hdr[2] = {world, active};
    // the marker count is per world in the batched kernel: pad with none
    if (report(cudaMemcpyAsync(r->d_markers, m, sizeof(float) * 4 * rd::kMaxMarkers, cudaMemcpyHostToDevice, st),
               "markers") ||
        report(cudaMemcpyAsync(r->d_ids, hdr, sizeof(hdr), cudaMemcpyHostToDevice, st), "ids"))
        return 0;
    const SimView sv = sim_view(s);
    if (render_any(r, s, r->d_ids, 1, n_markers ? r->d_markers : nullptr, n_markers, r->d_active, sv.n, r->d_rgb,
                   st) != ARC_OK)
        return 0;
    if (rgb) {
        const size_t bytes = (size_t)r->w * r->h * 3;
        if (report(cudaMemcpyAsync(r->h_scratch, r->d_rgb, bytes, cudaMemcpyDeviceToHost, st), "readback") ||
            report(cudaStreamSynchronize(st), "readback"))
            return 0;
        std::memcpy(rgb, r->h_scratch, bytes);
    } else if (report(cudaStreamSynchronize(st), "frame")) {
        return 0;
    }
    return 1;
}

void arc_render_size(const arc_renderer* r, int* width, int* height)
{
    if (width)
        *width = r ? r->w : 0;
    if (height)
        *height = r ? r->h : 0;
}

int arc_render_keys(arc_renderer*, int*, int) { return 0; }

void arc_render_set_title(arc_renderer*, const char*) {}

void arc_render_set_view(arc_renderer* r, int preset)
{
    static const double YAW[3] = {0.5, 1.4, 2.6};  // csrc/arc_render.c:962-968
    if (!r)
        return;
    r->view = ((preset % 3) + 3) % 3;
    r->yaw = YAW[r->view];
    r->pitch = 0.3;
}

int arc_render_set_samples(arc_renderer* r, int samples)
{
    if (!r || (samples != 1 && samples != 4))
        return ARC_ERR_ARG;
    r->samples = samples;
    return ARC_OK;
}

int arc_render_reset_cameras(arc_renderer* r)
{
    if (!r)
        return ARC_ERR_ARG;
    if (!r->d_cams)
        return ARC_OK;
    // after every call in flight, before any later one
    if (r->used && report(cudaEventSynchronize(r->done), "cameras"))
        return ARC_ERR_CUDA;
    if (report(cudaMemset(r->d_cams, 0, sizeof(rd::CamState) * (r->cam_n + 1)), "cameras") ||
        report(cudaDeviceSynchronize(), "cameras"))
        return ARC_ERR_CUDA;
    return ARC_OK;
}

int arc_render_frames(arc_renderer* r, const arc_sim* s, const int* d_ids, int n, const float* d_markers,
                      int markers_per_world, const int* d_active, unsigned char* d_rgb, void* stream)
{
    if (!r || !s || !d_rgb || n < 0 || markers_per_world < 0 || markers_per_world > rd::kMaxMarkers)
        return ARC_ERR_ARG;
    if (n == 0)
        return ARC_OK;
    if (!d_ids && n > arc_sim_num_worlds(s))
        return ARC_ERR_ARG;
    cudaStream_t st = stream ? (cudaStream_t)stream : (cudaStream_t)arc_sim_stream(s);
    return render_any(r, s, d_ids, n, d_markers, d_markers ? markers_per_world : 0, d_active, -1, d_rgb, st);
}

int arc_env_render(arc_renderer* r, const arc_sim* s, const int* d_ids, int n, unsigned char* d_rgb, void* stream)
{
    if (!r || !s || !d_rgb || n < 0)
        return ARC_ERR_ARG;
    TaskState ts;
    double radius = 0.0;
    if (!sim_task_view(s, &ts, &radius))
        return ARC_ERR_ARG;
    if (n == 0)
        return ARC_OK;
    if (!d_ids && n > arc_sim_num_worlds(s))
        return ARC_ERR_ARG;
    if (n > r->env_cap) {
        cudaFree(r->d_env_markers);
        cudaFree(r->d_env_active);
        r->d_env_markers = nullptr;
        r->d_env_active = nullptr;
        r->env_cap = 0;
        if (report(cudaMalloc((void**)&r->d_env_markers, sizeof(float) * 4 * n), "cudaMalloc(markers)") ||
            report(cudaMalloc((void**)&r->d_env_active, sizeof(int) * n), "cudaMalloc(markers)"))
            return ARC_ERR_CUDA;
        r->env_cap = n;
    }
    cudaStream_t st = stream ? (cudaStream_t)stream : (cudaStream_t)arc_sim_stream(s);
    rd::k_env_markers<<<(n + 127) / 128, 128, 0, st>>>(ts, radius, d_ids, n, r->d_env_markers, r->d_env_active);
    if (report(cudaGetLastError(), "env markers"))
        return ARC_ERR_CUDA;
    return render_any(r, s, d_ids, n, r->d_env_markers, 1, r->d_env_active, -1, d_rgb, st);
}

}  // extern "C"
