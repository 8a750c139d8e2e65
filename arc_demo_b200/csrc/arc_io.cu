// arc_io.cu - the reference ABI's read-out kernels (observe, heights,
// terrain lookups), state snapshots, and the FP64 reset with in-kernel
// terrain generation.
#include "arc_kernels.cuh"

namespace arc {

// ---------------------------------------------------------------------------
// csrc/arc_sim.c:140-183 (one thread per world)

template <class R>
__global__ void k_observe(const __grid_constant__ DevModel<R> M, Worlds<R> W, double* __restrict__ root,
                          double* __restrict__ rot, double* __restrict__ joints, double* __restrict__ contacts,
                          int* __restrict__ flags, const int* __restrict__ ids, int n_items)
{
    // output row k holds world ids[k] (world k without ids)
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_items)
        return;
    const int i = ids ? ids[k] : k;
    if (i < 0 || i >= W.n)
        return;
    const R* rec = W.rec + (size_t)i * W.stride;
    if (root) {
        double* r = root + (size_t)k * 13;
        for (int k = 0; k < 13; ++k)
            r[k] = (double)rec[k];
    }
    if (rot) {
        Q4<double> q{(double)rec[3], (double)rec[4], (double)rec[5], (double)rec[6]};
        M3<double> m = m3_from_quat(q);
        double* o = rot + (size_t)k * 9;
        for (int a = 0; a < 3; ++a)
            for (int c = 0; c < 3; ++c)
                o[a * 3 + c] = m.m[a][c];
    }
    if (joints) {
        const R* jr = rec + W.off_joint;
        double* o = joints + (size_t)k * 3 * M.nj;
        for (int j = 0; j < M.nj; ++j) {
            o[j] = (double)jr[j * kJointRec + 1];
            o[M.nj + j] = (double)jr[j * kJointRec + 2];
            o[2 * M.nj + j] = (double)jr[j * kJointRec + 3];
        }
    }
    if (contacts) {
        double* o = contacts + (size_t)k * M.n_channels;
        const double inv = 1.0 / M.substeps;
        const uint32_t* sph = W.sph + (size_t)i * M.ns;
        for (int c = 0; c < M.n_channels; ++c)
            o[c] = 0.0;
        for (int s = 0; s < M.ns; ++s) {
            double v = (int)(sph[s] & 0xffffu) * inv;
            double& c = o[M.channel[s]];
            c = c > v ? c : v;
        }
    }
    if (flags)
        flags[k] = W.unstable[i];
}

// Height of the column under (x, y) in FP64 (csrc/arc_terrain.h:42-50).
template <class R> __device__ __forceinline__ double terrain_height_d(const Worlds<R>& W, int i, double x, double y)
{
    const TerrainGeomD g = W.tgd[i];
    double fx = floor((x - g.ox) / g.cell), fy = floor((y - g.oy) / g.cell);
    if (!(fx >= 0.0 && fy >= 0.0 && fx < g.nx && fy < g.ny))
        return g.outside;
    if (!terrain_column_ok(W, i, (int)fx + (long long)(int)fy * g.nx, kCheckHeightsRead))
        return g.outside;
    return (double)W.th[W.toff[i] + (int)fx + (int)fy * g.nx];
}

// csrc/arc_sim.c:185-203 (one thread per sample)
template <class R>
__global__ void k_heights(Worlds<R> W, const double* __restrict__ offsets, int k, double* __restrict__ out)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)W.n * k)
        return;
    const int i = (int)(t / k), j = (int)(t % k);
    const R* rec = W.rec + (size_t)i * W.stride;
    V3<double> x{(double)rec[0], (double)rec[1], (double)rec[2]};
    Q4<double> q{(double)rec[3], (double)rec[4], (double)rec[5], (double)rec[6]};
    V3<double> fwd = qrotate(q, V3<double>{1.0, 0.0, 0.0});
    double yaw = atan2(fwd.y, fwd.x), c = cos(yaw), sn = sin(yaw);
    double f = offsets[2 * j], l = offsets[2 * j + 1];
    out[t] = terrain_height_d(W, i, x.x + c * f - sn * l, x.y + sn * f + c * l);
}

// csrc/arc_sim.c:205-210
template <class R>
__global__ void k_terrain_at(Worlds<R> W, const int* __restrict__ ids, const double* __restrict__ xy, int m,
                             double* __restrict__ out)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m)
        return;
    out[t] = terrain_height_d(W, ids[t], xy[2 * t], xy[2 * t + 1]);
}

// ---------------------------------------------------------------------------
// snapshots

template <class R>
__global__ void k_get_state(const __grid_constant__ DevModel<R> M, Worlds<R> W, const int* __restrict__ ids,
                            int n_ids, double* __restrict__ out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_ids)
        return;
    const int i = ids[k];
    const int stride = M.nb * 13 + M.ns * 8 + M.nj * 4 + 2;
    double* o = out + (size_t)k * stride;
    const R* rec = W.rec + (size_t)i * W.stride;
    for (int b = 0; b < M.nb * kBodyRec; ++b)
        *o++ = (double)rec[b];
    const R* sr = rec + W.off_sphere;
    const uint32_t* sph = W.sph + (size_t)i * M.ns;
    for (int s = 0; s < M.ns; ++s) {
        *o++ = (double)((sph[s] >> 16) & 1);
        for (int c = 0; c < 6; ++c)
            *o++ = (double)sr[s * kSphereRec + c];
        *o++ = (double)(sph[s] & 0xffffu);
    }
    const R* jr = rec + W.off_joint;
    for (int j = 0; j < M.nj * kJointRec; ++j)
        *o++ = (double)jr[j];
    *o++ = (double)W.unstable[i];
    *o++ = W.time[i];
}

template <class R>
__global__ void k_set_state(const __grid_constant__ DevModel<R> M, Worlds<R> W, const int* __restrict__ ids,
                            int n_ids, const double* __restrict__ in)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_ids)
        return;
    const int i = ids[k];
    const int stride = M.nb * 13 + M.ns * 8 + M.nj * 4 + 2;
    const double* p = in + (size_t)k * stride;
    R* rec = W.rec + (size_t)i * W.stride;
    for (int b = 0; b < M.nb * kBodyRec; ++b)
        rec[b] = (R)*p++;
    R* sr = rec + W.off_sphere;
    uint32_t* sph = W.sph + (size_t)i * M.ns;
    for (int s = 0; s < M.ns; ++s) {
        uint32_t anchored = *p++ != 0.0;
        for (int c = 0; c < 6; ++c)
            sr[s * kSphereRec + c] = (R)*p++;
        uint32_t touch = (uint32_t)*p++;
        sph[s] = (touch & 0xffffu) | (anchored << 16);
    }
    R* jr = rec + W.off_joint;
    for (int j = 0; j < M.nj * kJointRec; ++j)
        jr[j] = (R)*p++;
    W.unstable[i] = *p++ != 0.0;
    W.time[i] = *p++;
}

// ---------------------------------------------------------------------------
// RNG (csrc/arc_rng.h:14-53), integer exact

struct Rng {
    uint32_t s[4];
};

__device__ __forceinline__ uint32_t rng_u32(Rng& r)
{
    uint32_t t = r.s[3], s = r.s[0];
    r.s[3] = r.s[2];
    r.s[2] = r.s[1];
    r.s[1] = s;
    t = t ^ (t << 11);
    t ^= t >> 8;
    r.s[0] = t ^ s ^ (s >> 19);
    return r.s[0];
}

__device__ __forceinline__ uint32_t hash32(uint32_t x)
{
    x = (x ^ (x >> 16)) * 0x7feb352dU;
    x = (x ^ (x >> 15)) * 0x846ca68bU;
    return x ^ (x >> 16);
}

__device__ __forceinline__ void rng_seed(Rng& r, uint32_t seed)
{
    for (int i = 0; i < 4; ++i) {
        seed = hash32(seed + 0x9e3779b9U * (uint32_t)(i + 1));
        r.s[i] = seed ? seed : 1U;
    }
}

__device__ __forceinline__ double rng_range(Rng& r, double lo, double hi)
{
    return lo + (hi - lo) * (rng_u32(r) * (1.0 / 4294967296.0));
}

// ---------------------------------------------------------------------------
// reset (csrc/arc_sim.c:88-110 + csrc/arc_terrain.c:35-71 + csrc/arc_phys.c:749-782)

__device__ __forceinline__ double smooth(double t) { return t * t * (3.0 - 2.0 * t); }

// value noise of one octave at column (ix, iy) (csrc/arc_terrain.c:38-56)
__device__ __forceinline__ double noise_at(const double* lat, int m, int spacing, int ix, int iy)
{
    double fx = (double)ix / spacing, fy = (double)iy / spacing;
    int gx = (int)fx, gy = (int)fy;
    double tx = smooth(fx - gx), ty = smooth(fy - gy);
    double a = lat[gx + gy * m], b = lat[gx + 1 + gy * m];
    double c = lat[gx + (gy + 1) * m], d = lat[gx + 1 + (gy + 1) * m];
    return (a + (b - a) * tx) * (1.0 - ty) + (c + (d - c) * tx) * ty;
}

// Column cells hit by the reset's footprint scan (csrc/arc_sim.c:104-107):
// a 64-bit mask of in-range cells plus whether any sample fell outside.
__device__ __forceinline__ unsigned long long scan_cells(double reach, double step, double o, double cell, int n,
                                                         bool& outside)
{
    unsigned long long mask = 0;
    for (double x = -reach; x <= reach; x += step) {
        double f = floor((x - o) / cell);
        if (f >= 0.0 && f < n)
            mask |= 1ull << (int)f;
        else
            outside = true;
    }
    return mask;
}

template <class R>
__global__ void k_reset(const __grid_constant__ ResetModel RM, Worlds<R> W, TerrainGeom<R>* tg, TerrainGeomD* tgd,
                        const int* __restrict__ ids, int n_ids, const unsigned* __restrict__ seeds,
                        const double* __restrict__ difficulty, const int* __restrict__ grid_of, double cell)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_ids)
        return;
    const int i = ids[k];
    const double diff = difficulty[k];
    int n = grid_of ? grid_of[i] : 64;
    n = n < kGridMax ? n : kGridMax;
    Rng rng;
    rng_seed(rng, seeds[k]);

    // geometry (csrc/arc_terrain.c:17-30 with outside = void)
    TerrainGeomD g;
    g.nx = g.ny = n;
    g.cell = cell;
    g.ox = -0.5 * n * cell;
    g.oy = -0.5 * n * cell;
    g.outside = -100.0;
    tgd[i] = g;
    tg[i] = TerrainGeom<R>{n, n, (R)g.cell, (R)g.ox, (R)g.oy, (R)g.outside};
    R* h = W.th + W.toff[i];
    if (!terrain_column_ok(W, i, (long long)n * n - 1, kCheckTerrainWrite))
        return;

    const double reach = RM.footprint + 0.1, step = 0.5 * cell;
    bool out_x = false, out_y = false;
    const unsigned long long mx = scan_cells(reach, step, g.ox, cell, n, out_x);
    const unsigned long long my = scan_cells(reach, step, g.oy, cell, n, out_y);
    double ground = -1e30;
    if (out_x || out_y)
        ground = g.outside;

    if (diff <= 0.0) {
        for (int c = 0; c < n * n; ++c)
            h[c] = R(0);
        if (mx && my)
            ground = ground > 0.0 ? ground : 0.0;
    } else {
        double lat1[(kGridMax / 8 + 2) * (kGridMax / 8 + 2)];
        double lat2[(kGridMax / 3 + 2) * (kGridMax / 3 + 2)];
        const int m1 = n / 8 + 2, m2 = n / 3 + 2;
        for (int c = 0; c < m1 * m1; ++c)
            lat1[c] = rng_range(rng, -1.0, 1.0);
        for (int c = 0; c < m2 * m2; ++c)
            lat2[c] = rng_range(rng, -1.0, 1.0);
        const double amp1 = 0.45 * diff, amp2 = 0.12 * diff, ampj = 0.06 * diff;
        // origin column, whose height becomes 0 (csrc/arc_terrain.c:68-70)
        const double f0x = floor((0.0 - g.ox) / g.cell), f0y = floor((0.0 - g.oy) / g.cell);
        const bool base_in = f0x >= 0.0 && f0y >= 0.0 && f0x < n && f0y < n;
        const int c0 = base_in ? (int)f0x + (int)f0y * n : -1;
        // pass 1: the quantised height of the origin column
        const Rng saved = rng;
        double base = g.outside;
        if (base_in) {
            for (int c = 0; c < c0; ++c)
                rng_u32(rng);
            const int ix = c0 % n, iy = c0 / n;
            double v = amp1 * noise_at(lat1, m1, 8, ix, iy);
            v = v + amp2 * noise_at(lat2, m2, 3, ix, iy);
            double hj = v + ampj * rng_range(rng, -1.0, 1.0);
            base = 0.03 * floor(hj / 0.03 + 0.5);
        }
        // pass 2: every column, shifted by the base
        rng = saved;
        double gmax = -1e300;
        for (int iy = 0; iy < n; ++iy)
            for (int ix = 0; ix < n; ++ix) {
                double v = amp1 * noise_at(lat1, m1, 8, ix, iy);
                v = v + amp2 * noise_at(lat2, m2, 3, ix, iy);
                double hj = v + ampj * rng_range(rng, -1.0, 1.0);
                double hf = 0.03 * floor(hj / 0.03 + 0.5) - base;
                h[ix + iy * n] = (R)hf;
                if (((mx >> ix) & 1) && ((my >> iy) & 1))
                    gmax = gmax > hf ? gmax : hf;
            }
        if (mx && my)
            ground = ground > gmax ? ground : gmax;
    }

    // noisy stance and yaw (csrc/arc_sim.c:99-102)
    double angles[kMaxJoints];
    for (int j = 0; j < RM.nj; ++j) {
        double a = RM.default_angles[j] + rng_range(rng, -0.1, 0.1);
        angles[j] = a < RM.lo[j] ? RM.lo[j] : (a > RM.hi[j] ? RM.hi[j] : a);
    }
    const double yaw = rng_range(rng, -kPi, kPi);

    // forward kinematics (csrc/arc_phys.c:749-767)
    V3<double> xs[kMaxBodies];
    Q4<double> qs[kMaxBodies];
    const double hy = sin(0.5 * yaw), cy = cos(0.5 * yaw);
    xs[0] = V3<double>{0.0, 0.0, ground + RM.stand_height + 0.03};
    qs[0] = qnormalize(Q4<double>{cy, 0.0 * hy, 0.0 * hy, 1.0 * hy});
    for (int j = 0; j < RM.nj; ++j) {
        const int p = RM.parent[j], c = RM.child[j];
        V3<double> xp = p >= 0 ? xs[p] : V3<double>{0.0, 0.0, 0.0};
        Q4<double> qp = p >= 0 ? qs[p] : q_identity<double>();
        V3<double> anchor = xp + qrotate(qp, RM.r1[j]);
        const double s = sin(0.5 * angles[j]), ca = cos(0.5 * angles[j]);
        Q4<double> qa{ca, RM.a1[j].x * s, RM.a1[j].y * s, RM.a1[j].z * s};
        qs[c] = qnormalize(qmul(qp, qmul(qa, RM.q_rel0[j])));
        xs[c] = anchor - qrotate(qs[c], RM.r2[j]);
    }

    R* rec = W.rec + (size_t)i * W.stride;
    for (int b = 0; b < RM.nb; ++b) {
        R* r = rec + b * kBodyRec;
        r[0] = (R)xs[b].x; r[1] = (R)xs[b].y; r[2] = (R)xs[b].z;
        r[3] = (R)qs[b].w; r[4] = (R)qs[b].x; r[5] = (R)qs[b].y; r[6] = (R)qs[b].z;
        for (int c = 7; c < 13; ++c)
            r[c] = R(0);
    }
    R* sr = rec + W.off_sphere;
    uint32_t* sph = W.sph + (size_t)i * RM.ns;
    for (int s = 0; s < RM.ns; ++s) {
        for (int c = 0; c < kSphereRec; ++c)
            sr[s * kSphereRec + c] = R(0);
        sph[s] = 0;
    }
    R* jr = rec + W.off_joint;
    for (int j = 0; j < RM.nj; ++j) {
        jr[j * kJointRec + 0] = (R)angles[j];
        jr[j * kJointRec + 1] = (R)angles[j];
        jr[j * kJointRec + 2] = R(0);
        jr[j * kJointRec + 3] = R(0);
    }
    W.unstable[i] = 0;
    W.time[i] = 0.0;
}

template <class R>
__global__ void k_set_terrain(Worlds<R> W, TerrainGeom<R>* tg, TerrainGeomD* tgd, int id, int nx, int ny, double cell,
                              double outside, const double* __restrict__ heights)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0) {
        TerrainGeomD g{nx, ny, cell, -0.5 * nx * cell, -0.5 * ny * cell, outside};
        tgd[id] = g;
        tg[id] = TerrainGeom<R>{nx, ny, (R)g.cell, (R)g.ox, (R)g.oy, (R)g.outside};
    }
    if (t < nx * ny && terrain_column_ok(W, id, t, kCheckTerrainWrite))
        W.th[W.toff[id] + t] = (R)heights[t];
}

// ---------------------------------------------------------------------------
// launchers

static inline int blocks_for(long long n, int threads) { return (int)((n + threads - 1) / threads); }

template <class R>
cudaError_t launch_observe(const DevModel<R>& M, const Worlds<R>& W, double* root, double* rot, double* joints,
                           double* contacts, int* flags, cudaStream_t stream, const int* ids, int n_items)
{
    if (!ids)
        n_items = W.n;
    if (W.n <= 0 || n_items <= 0)
        return cudaSuccess;
    k_observe<R><<<blocks_for(n_items, 128), 128, 0, stream>>>(M, W, root, rot, joints, contacts, flags, ids,
                                                               n_items);
    return cudaGetLastError();
}

template <class R>
cudaError_t launch_heights(const Worlds<R>& W, const double* offsets, int k, double* out, cudaStream_t stream)
{
    if (W.n <= 0 || k <= 0)
        return cudaSuccess;
    k_heights<R><<<blocks_for((long long)W.n * k, 256), 256, 0, stream>>>(W, offsets, k, out);
    return cudaGetLastError();
}

template <class R>
cudaError_t launch_terrain_at(const Worlds<R>& W, const int* ids, const double* xy, int m, double* out,
                              cudaStream_t stream)
{
    if (m <= 0)
        return cudaSuccess;
    k_terrain_at<R><<<blocks_for(m, 128), 128, 0, stream>>>(W, ids, xy, m, out);
    return cudaGetLastError();
}

template <class R>
cudaError_t launch_get_state(const DevModel<R>& M, const Worlds<R>& W, const int* ids, int n_ids, double* out,
                             cudaStream_t stream)
{
    if (n_ids <= 0)
        return cudaSuccess;
    k_get_state<R><<<blocks_for(n_ids, 128), 128, 0, stream>>>(M, W, ids, n_ids, out);
    return cudaGetLastError();
}

template <class R>
cudaError_t launch_set_state(const DevModel<R>& M, const Worlds<R>& W, const int* ids, int n_ids, const double* in,
                             cudaStream_t stream)
{
    if (n_ids <= 0)
        return cudaSuccess;
    k_set_state<R><<<blocks_for(n_ids, 128), 128, 0, stream>>>(M, W, ids, n_ids, in);
    return cudaGetLastError();
}

template <class R>
cudaError_t launch_reset(const ResetModel& RM, const Worlds<R>& W, TerrainGeom<R>* tg, TerrainGeomD* tgd,
                         const int* ids, int n_ids, const unsigned* seeds, const double* difficulty,
                         const int* grid_of, double cell, cudaStream_t stream)
{
    if (n_ids <= 0)
        return cudaSuccess;
    k_reset<R><<<blocks_for(n_ids, 64), 64, 0, stream>>>(RM, W, tg, tgd, ids, n_ids, seeds, difficulty, grid_of,
                                                        cell);
    return cudaGetLastError();
}

template <class R>
cudaError_t launch_set_terrain(const Worlds<R>& W, TerrainGeom<R>* tg, TerrainGeomD* tgd, int id, int nx, int ny,
                               double cell, double outside, const double* heights, cudaStream_t stream)
{
    k_set_terrain<R><<<blocks_for(nx * ny > 0 ? nx * ny : 1, 256), 256, 0, stream>>>(W, tg, tgd, id, nx, ny, cell,
                                                                                    outside, heights);
    return cudaGetLastError();
}

#define ARC_INSTANTIATE_IO(R)                                                                                      \
    template cudaError_t launch_observe<R>(const DevModel<R>&, const Worlds<R>&, double*, double*, double*,      \
                                           double*, int*, cudaStream_t, const int*, int);                        \
    template cudaError_t launch_heights<R>(const Worlds<R>&, const double*, int, double*, cudaStream_t);          \
    template cudaError_t launch_terrain_at<R>(const Worlds<R>&, const int*, const double*, int, double*,          \
                                              cudaStream_t);                                                     \
    template cudaError_t launch_get_state<R>(const DevModel<R>&, const Worlds<R>&, const int*, int, double*,     \
                                             cudaStream_t);                                                      \
    template cudaError_t launch_set_state<R>(const DevModel<R>&, const Worlds<R>&, const int*, int,              \
                                             const double*, cudaStream_t);                                       \
    template cudaError_t launch_reset<R>(const ResetModel&, const Worlds<R>&, TerrainGeom<R>*, TerrainGeomD*,    \
                                         const int*, int, const unsigned*, const double*, const int*, double,    \
                                         cudaStream_t);                                                          \
    template cudaError_t launch_set_terrain<R>(const Worlds<R>&, TerrainGeom<R>*, TerrainGeomD*, int, int, int,  \
                                               double, double, const double*, cudaStream_t);

ARC_INSTANTIATE_IO(float)
ARC_INSTANTIATE_IO(double)

}  // namespace arc
