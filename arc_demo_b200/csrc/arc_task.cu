// arc_task.cu - task layer kernels (arc/task.py on the device) and the
// warp-cooperative world reset (csrc/arc_sim.c:88-110).
#include "arc_task.cuh"
#include "arc_step_warps.cuh"

namespace arc {

namespace {

// ---------------------------------------------------------------------------
// reference RNG (csrc/arc_rng.h:14-53), integer exact

struct Xorshift {
    uint32_t s[4];
    __device__ __forceinline__ uint32_t next()
    {
        uint32_t t = s[3], v = s[0];
        s[3] = s[2];
        s[2] = s[1];
        s[1] = v;
        t = t ^ (t << 11);
        t ^= t >> 8;
        s[0] = t ^ v ^ (v >> 19);
        return s[0];
    }
    __device__ __forceinline__ void seed(uint32_t seed)
    {
        for (int i = 0; i < 4; ++i) {
            uint32_t x = seed + 0x9e3779b9U * (uint32_t)(i + 1);
            x = (x ^ (x >> 16)) * 0x7feb352dU;
            x = (x ^ (x >> 15)) * 0x846ca68bU;
            seed = x ^ (x >> 16);
            s[i] = seed ? seed : 1U;
        }
    }
};

// Jumping ahead in the stream. xorshift128 is linear over GF(2): one step
// is a 128 x 128 bit matrix M acting on the state (s0 s1 s2 s3). Column b
// of M^(2^k), for k < kJumpBits, is g_jump[k][b] (built once per device by
// k_jump_init), so skipping d draws costs one XOR of a column per set state
// bit, for each set bit of d; the draws that follow are the stream's own,
// bit for bit.
constexpr int kJumpBits = 13;  // skips below 8,192 draws (a 64 x 64 terrain takes 4,742)
__device__ uint4 g_jump[kJumpBits][128];

__global__ void k_jump_init()
{
    const int k = blockIdx.x, b = threadIdx.x;
    Xorshift r;
    for (int w = 0; w < 4; ++w)
        r.s[w] = (b >> 5) == w ? 1u << (b & 31) : 0u;
    for (int it = 0; it < (1 << k); ++it)
        r.next();
    g_jump[k][b] = make_uint4(r.s[0], r.s[1], r.s[2], r.s[3]);
}

__device__ __forceinline__ void rng_skip(Xorshift& r, uint32_t d)
{
    for (int k = 0; d; ++k, d >>= 1) {
        if (!(d & 1u))
            continue;
        uint32_t o[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (int w = 0; w < 4; ++w) {
            uint32_t bits = r.s[w];
            while (bits) {
                const int b = __ffs(bits) - 1;
                bits &= bits - 1u;
                const uint4 c = g_jump[k][w * 32 + b];
                o[0] ^= c.x;
                o[1] ^= c.y;
                o[2] ^= c.z;
                o[3] ^= c.w;
            }
        }
#pragma unroll
        for (int w = 0; w < 4; ++w)
            r.s[w] = o[w];
    }
}

// rng_range(lo, hi) of a raw draw u (csrc/arc_rng.h:45-53)
__device__ __forceinline__ double range_of(uint32_t u, double lo, double hi)
{
    return lo + (hi - lo) * (u * (1.0 / 4294967296.0));
}

// ---------------------------------------------------------------------------
// device RNG of the task layer (checkpoints, reset seeds): a counter-based
// splitmix64 stream per (seed, world, kind). The reference draws these from
// numpy's PCG64 on the host (arc/task.py:117,138-139); the device cannot
// reproduce that stream, so it draws the same distributions from its own.

__device__ __forceinline__ uint64_t splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

__device__ __forceinline__ uint64_t stream_u64(uint64_t seed, int world, uint32_t kind, uint32_t counter)
{
    return splitmix64(splitmix64(seed ^ (((uint64_t)(uint32_t)world << 32) | kind)) + counter);
}

__device__ __forceinline__ double unit(uint64_t x) { return (double)(x >> 11) * (1.0 / 9007199254740992.0); }

// the identity of world i's streams: its index, or the key its tenant gave it
__device__ __forceinline__ int key_of(const TaskState& S, int i) { return S.key ? (int)S.key[i] : i; }

// ---------------------------------------------------------------------------
// world read-out in FP64 (what arc_sim_observe returns, csrc/arc_sim.c:140-183)

struct Obs64 {
    V3<double> x, v, w;
    Q4<double> q;
    M3<double> rot;
    double angle[kNumJoints], rate[kNumJoints], torque[kNumJoints];
    double contact[kNumLegs + 2];
    int unstable;
};

template <class R>
__device__ void read_world(const DevModel<R>& M, const Worlds<R>& W, int i, Obs64& o)
{
    const R* rec = W.rec + (size_t)i * W.stride;
    o.x = V3<double>{(double)rec[0], (double)rec[1], (double)rec[2]};
    o.q = Q4<double>{(double)rec[3], (double)rec[4], (double)rec[5], (double)rec[6]};
    o.v = V3<double>{(double)rec[7], (double)rec[8], (double)rec[9]};
    o.w = V3<double>{(double)rec[10], (double)rec[11], (double)rec[12]};
    o.rot = m3_from_quat(o.q);
    const R* jr = rec + W.off_joint;
    for (int j = 0; j < kNumJoints; ++j) {
        o.angle[j] = (double)jr[j * kJointRec + 1];
        o.rate[j] = (double)jr[j * kJointRec + 2];
        o.torque[j] = (double)jr[j * kJointRec + 3];
    }
    const uint32_t* sph = W.sph + (size_t)i * M.ns;
    const double inv = 1.0 / M.substeps;
    for (int c = 0; c < kNumLegs + 2; ++c)
        o.contact[c] = 0.0;
    for (int s = 0; s < M.ns; ++s) {
        double v = (int)(sph[s] & 0xffffu) * inv;
        double& c = o.contact[M.channel[s]];
        c = c > v ? c : v;
    }
    o.unstable = W.unstable[i];
}

template <class R> __device__ __forceinline__ double height_at(const Worlds<R>& W, int i, double x, double y)
{
    const TerrainGeomD g = W.tgd[i];
    double fx = floor((x - g.ox) / g.cell), fy = floor((y - g.oy) / g.cell);
    if (!(fx >= 0.0 && fy >= 0.0 && fx < g.nx && fy < g.ny))
        return g.outside;
    if (!terrain_column_ok(W, i, (int)fx + (long long)(int)fy * g.nx, kCheckHeightsRead))
        return g.outside;
    return (double)W.th[W.toff[i] + (int)fx + (int)fy * g.nx];
}

// |angle| between the gaze (body +x on the ground) and the target (arc/task.py:79-85)
__device__ __forceinline__ double gaze_error(const M3<double>& rot, V3<double> pos, const double* target)
{
    double fx = rot.m[0][0], fy = rot.m[1][0];
    double dx = target[0] - pos.x, dy = target[1] - pos.y;
    return fabs(atan2(fx * dy - fy * dx, fx * dx + fy * dy));
}

// R^T a, summed like numpy's a @ R for a row vector
__device__ __forceinline__ V3<double> rt_mul(const M3<double>& r, V3<double> a)
{
    return V3<double>{a.x * r.m[0][0] + a.y * r.m[1][0] + a.z * r.m[2][0],
                      a.x * r.m[0][1] + a.y * r.m[1][1] + a.z * r.m[2][1],
                      a.x * r.m[0][2] + a.y * r.m[1][2] + a.z * r.m[2][2]};
}

__device__ __forceinline__ float obs_value(double v)
{
    float f = (float)v;
    return isfinite(f) ? f : 0.0f;
}

// arc/task.py:231-259: writes the 195 observation values of world i
// Observation entries m_begin .. m_end - 1 of the 143 terrain heights in the
// heading frame (csrc/arc_sim.c:185-203), written to dst[m - m_begin], kChunk
// samples at a time: their terrain loads are all issued before any is used.
template <int kChunk, class R>
__device__ void write_heights(const TaskParams& P, const Worlds<R>& W, int i, V3<double> x, Q4<double> q, float* dst,
                              int m_begin, int m_end)
{
    V3<double> f = qrotate(q, V3<double>{1.0, 0.0, 0.0});
    const double yaw = atan2(f.y, f.x), cy = cos(yaw), sy = sin(yaw);
    const TerrainGeomD g = W.tgd[i];
    const R* th = W.th + W.toff[i];
    int k = 0;
    for (int m0 = m_begin; m0 < m_end; m0 += kChunk) {
        double h[kChunk];
#pragma unroll
        for (int u = 0; u < kChunk; ++u) {
            const int m = m0 + u < m_end ? m0 + u : m_end - 1;
            const double fo = P.offsets[m][0], lo = P.offsets[m][1];
            const double px = x.x + cy * fo - sy * lo, py = x.y + sy * fo + cy * lo;
            // csrc/arc_terrain.h:42-50
            const double fx = floor((px - g.ox) / g.cell), fy = floor((py - g.oy) / g.cell);
            const bool in = fx >= 0.0 && fy >= 0.0 && fx < g.nx && fy < g.ny &&
                            terrain_column_ok(W, i, (int)fx + (long long)(int)fy * g.nx, kCheckHeightsRead);
            const int idx = in ? (int)fx + (int)fy * g.nx : 0;
            const double top = (double)__ldg(th + idx);
            h[u] = in ? top : g.outside;
        }
#pragma unroll
        for (int u = 0; u < kChunk; ++u) {
            if (m0 + u >= m_end)
                break;
            double rel = x.z - P.stand_height - h[u];
            rel = rel < -1.0 ? -1.0 : (rel > 1.0 ? 1.0 : rel);
            dst[k++] = obs_value(rel);
        }
    }
}

template <class R>
__device__ void write_obs(const TaskParams& P, const Worlds<R>& W, const TaskState& S, int i, const Obs64& o,
                          float* dst, bool heights = true)
{
    const M3<double>& r = o.rot;
    int k = 0;
    dst[k++] = obs_value(-r.m[2][0]);
    dst[k++] = obs_value(-r.m[2][1]);
    dst[k++] = obs_value(-r.m[2][2]);
    V3<double> lin = rt_mul(r, o.v), ang = rt_mul(r, o.w);
    dst[k++] = obs_value(lin.x);
    dst[k++] = obs_value(lin.y);
    dst[k++] = obs_value(lin.z);
    dst[k++] = obs_value(0.25 * ang.x);
    dst[k++] = obs_value(0.25 * ang.y);
    dst[k++] = obs_value(0.25 * ang.z);
    for (int j = 0; j < kNumJoints; ++j)
        dst[k++] = obs_value(o.angle[j] - P.default_angles[j]);
    for (int j = 0; j < kNumJoints; ++j)
        dst[k++] = obs_value(0.1 * o.rate[j]);
    for (int j = 0; j < kNumJoints; ++j)
        dst[k++] = obs_value((double)S.prev_action[(size_t)i * kNumJoints + j]);
    const double heading = atan2(r.m[1][0], r.m[0][0]);
    const double dx = S.target[2 * i] - o.x.x, dy = S.target[2 * i + 1] - o.x.y;
    const double c = cos(heading), s = sin(heading);
    const double fwd = c * dx + s * dy, left = -s * dx + c * dy;
    double dist = hypot(fwd, left);
    dist = dist > 1e-6 ? dist : 1e-6;
    dst[k++] = obs_value(fwd / dist);
    dst[k++] = obs_value(left / dist);
    dst[k++] = obs_value((dist < 6.0 ? dist : 6.0) / 6.0);
    if (heights)
        write_heights<8>(P, W, i, o.x, o.q, dst + k, 0, kNumOffsets);
    k += kNumOffsets;
    for (int l = 0; l < kNumLegs; ++l)
        dst[k++] = obs_value(o.contact[l]);
}

// Checkpoint 3-6 m away inside the terrain (arc/task.py:127-151), drawn
// from the device stream; also refreshes target_z, prev_dist, prev_gaze.
template <class R>
__device__ void place_target(const TaskParams& P, const Worlds<R>& W, const TaskState& S, int i, V3<double> pos,
                             const M3<double>& rot)
{
    const double limit = P.half_extent - P.border;
    double tx = 0.5 * pos.x, ty = 0.5 * pos.y;
    for (int t = 0; t < 20; ++t) {
        const unsigned k = S.draws[i]++;
        const double ang = -kPi + 2.0 * kPi * unit(stream_u64(P.seed, key_of(S, i), 1u, 2u * k));
        const double dist = P.checkpoint_min_dist +
                            (P.checkpoint_max_dist - P.checkpoint_min_dist) *
                                unit(stream_u64(P.seed, key_of(S, i), 1u, 2u * k + 1u));
        const double cx = pos.x + dist * cos(ang), cy = pos.y + dist * sin(ang);
        if (fabs(cx) < limit && fabs(cy) < limit) {
            tx = cx;
            ty = cy;
            break;
        }
    }
    S.target[2 * i] = tx;
    S.target[2 * i + 1] = ty;
    S.target_z[i] = height_at(W, i, tx, ty);
    const double dx = tx - pos.x, dy = ty - pos.y;
    S.prev_dist[i] = sqrt(dx * dx + dy * dy);
    S.prev_gaze[i] = gaze_error(rot, pos, S.target + 2 * i);
    S.in_view[i] = S.prev_gaze[i] < P.fov_rad;
}

// ---------------------------------------------------------------------------
// arc/task.py:155-220 (+ 231-259 for the observation): one thread per world

// One world's step of the task layer; returns whether its episode ended.
// Compiled once (not inlined): the separate task kernel and the fused
// control step run the same code.
template <class R>
__device__ __noinline__ bool task_step_world(const DevModel<R>& M, const Worlds<R>& W, const TaskParams& P, const TaskState& S,
                                const TaskOut& O, const float* __restrict__ actions, int write_obs_rows, int i)
{
    Obs64 o;
    read_world(M, W, i, o);
    const int steps = S.steps[i] + 1;
    S.steps[i] = steps;
    const double* tgt = S.target + 2 * i;
    const double dist = hypot(tgt[0] - o.x.x, tgt[1] - o.x.y);
    const double gaze = gaze_error(o.rot, o.x, tgt);
    double view = (cos(gaze) - P.cos_fov) / (1.0 - P.cos_fov);
    view = view < 0.0 ? 0.0 : (view > 1.0 ? 1.0 : view);
    const bool in_view = gaze < P.fov_rad;
    double progress = S.prev_dist[i] - dist;
    progress = progress < P.max_speed * P.dt ? progress : P.max_speed * P.dt;
    if (progress > 0)
        progress = progress * view;
    const double turn = S.prev_gaze[i] - gaze;
    const bool reached = dist < P.checkpoint_radius && in_view;
    const V3<double> br = rt_mul(o.rot, o.w);
    const bool torso = o.contact[kNumLegs] > 0;
    const int torso_steps = torso ? S.torso_steps[i] + 1 : 0;
    S.torso_steps[i] = torso_steps;
    double power = 0.0, rate = 0.0;
    float* pa = S.prev_action + (size_t)i * kNumJoints;
    for (int j = 0; j < kNumJoints; ++j) {
        power += fabs(o.rate[j] * o.torque[j]);
        double a = (double)actions[(size_t)i * kNumJoints + j];
        a = a < -1.0 ? -1.0 : (a > 1.0 ? 1.0 : a);
        const double d = a - (double)pa[j];
        rate += d * d;
        pa[j] = (float)a;
    }
    double reward = P.w_progress * progress + P.w_turn * turn + P.w_checkpoint * (reached ? 1.0 : 0.0) - P.w_time -
                    P.w_energy * power * P.dt - P.w_action_rate * rate -
                    P.w_body_contact * (o.contact[kNumLegs + 1] > 0 ? 1.0 : 0.0) -
                    P.w_torso_contact * (torso ? 1.0 : 0.0) - P.w_body_rate * (br.x * br.x + br.y * br.y) -
                    P.w_bounce * (o.v.z * o.v.z);
    bool finite = true;
    {
        const double r13[13] = {o.x.x, o.x.y, o.x.z, o.q.w, o.q.x, o.q.y, o.q.z,
                                o.v.x, o.v.y, o.v.z, o.w.x, o.w.y, o.w.z};
        for (int c = 0; c < 13; ++c)
            finite = finite && isfinite(r13[c]);
    }
    const bool bad = o.unstable != 0 || !finite;
    const bool vd = fabs(o.x.x) > P.half_extent || fabs(o.x.y) > P.half_extent || o.x.z < P.void_z;
    const bool flip = o.rot.m[2][2] < P.flip_up_z;
    const bool beached = torso_steps > P.beached_steps;
    const bool fell = flip || beached || vd || bad;
    const int cause = bad ? 1 : (vd ? 2 : (flip ? 3 : (beached ? 4 : 0)));
    if (fell)
        reward = reward - P.w_fall;
    if (bad)
        reward = -P.w_fall;
    S.prev_dist[i] = dist;
    S.prev_gaze[i] = gaze;
    S.in_view[i] = in_view;
    const int checkpoints = S.checkpoints[i] + (reached ? 1 : 0);
    S.checkpoints[i] = checkpoints;
    if (reached && !fell)
        place_target(P, W, S, i, o.x, o.rot);
    const bool truncated = steps >= P.max_steps && !fell;
    O.reward[i] = (float)reward;
    O.terminated[i] = fell;
    O.truncated[i] = truncated;
    O.cause[i] = (signed char)cause;
    const bool done = fell || truncated;
    if (done) {
        O.ended_checkpoints[i] = checkpoints;
        O.ended_difficulty[i] = S.difficulty[i];
        O.ended_steps[i] = steps;
        if (P.curriculum) {
            // arc/task.py:222-227
            const bool up = checkpoints >= P.level_up_checkpoints;
            const bool down = fell && checkpoints == 0 && steps < P.level_down_steps;
            double lvl = S.level[i] + P.level_step * ((up ? 1.0 : 0.0) - (down ? 1.0 : 0.0));
            lvl = rint(lvl * 1e6) / 1e6;
            S.level[i] = lvl < 0.0 ? 0.0 : (lvl > P.max_difficulty ? P.max_difficulty : lvl);
        }
        if (O.done_list)
            O.done_list[atomicAdd(O.done_count, 1)] = i;
    }
    if (write_obs_rows && O.obs) {
        float* row = O.obs + (size_t)i * kObsSize;
        write_obs(P, W, S, i, o, row, write_obs_rows == 1);
        if (done && O.terminal_obs) {
            float* t = O.terminal_obs + (size_t)i * kObsSize;
            for (int k = 0; k < kObsSize; ++k)
                t[k] = row[k];
        }
    }
    return done;
}

// Worlds first + k (or ids[k]) for k < count, one thread each.
template <class R>
__global__ void k_task_step(const __grid_constant__ DevModel<R> M, Worlds<R> W, const __grid_constant__ TaskParams P,
                            TaskState S, TaskOut O, const float* __restrict__ actions, int write_obs_rows, int first,
                            int count, const int* __restrict__ ids)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count)
        return;
    task_step_world(M, W, P, S, O, actions, write_obs_rows, ids ? ids[k] : first + k);
}

// The observations' terrain heights of worlds first .. first + count - 1,
// kHeightsPer samples per thread (k_task_step, with write_obs_rows == 2,
// writes the rest of each row): the 143 samples of a world spread over nine
// threads instead of one, four loads in flight per thread and registers sized
// for eight blocks per SM (the kernel waits on latency: occupancy pays more
// than loads in flight). Rows of worlds that ended this step get them in
// their terminal observation too.
constexpr int kHeightsPer = 16;
constexpr int kHeightParts = (kNumOffsets + kHeightsPer - 1) / kHeightsPer;
constexpr int kHeightsAt = 9 + 3 * kNumJoints + 3;  // offset of the heights in a row

constexpr int kHeightThreads = 128;
constexpr int kHeightBlocks = 8;

// Part `part` (kHeightsPer samples) of world i's observation heights
// (compiled once, as task_step_world).
template <class R>
__device__ __noinline__ void task_heights_part(const Worlds<R>& W, const TaskParams& P, const TaskOut& O, int i,
                                                  int part)
{
    const int m0 = part * kHeightsPer, m1 = m0 + kHeightsPer < kNumOffsets ? m0 + kHeightsPer : kNumOffsets;
    const R* b0 = W.rec + (size_t)i * W.stride;  // the torso's pose, as read_world reads it
    const V3<double> x{(double)b0[0], (double)b0[1], (double)b0[2]};
    const Q4<double> q{(double)b0[3], (double)b0[4], (double)b0[5], (double)b0[6]};
    float* row = O.obs + (size_t)i * kObsSize + kHeightsAt;
    write_heights<4>(P, W, i, x, q, row + m0, m0, m1);
    if (O.terminal_obs && (O.terminated[i] | O.truncated[i])) {
        float* t_row = O.terminal_obs + (size_t)i * kObsSize + kHeightsAt;
        for (int m = m0; m < m1; ++m)
            t_row[m] = row[m];
    }
}

template <class R>
__global__ void __launch_bounds__(kHeightThreads, kHeightBlocks)
    k_task_heights(const __grid_constant__ DevModel<R> M, Worlds<R> W, const __grid_constant__ TaskParams P, TaskOut O,
                   int first, int count, const int* __restrict__ ids)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)count * kHeightParts)
        return;
    const int k = (int)(t / kHeightParts);
    task_heights_part(W, P, O, ids ? ids[k] : first + k, (int)(t % kHeightParts));
}

template <class R>
__global__ void k_task_observe(const __grid_constant__ DevModel<R> M, Worlds<R> W, const __grid_constant__ TaskParams P,
                               TaskState S, float* obs, const int* __restrict__ ids, int n)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    const int i = ids ? ids[k] : k;
    Obs64 o;
    read_world(M, W, i, o);
    write_obs(P, W, S, i, o, obs + (size_t)i * kObsSize);
}

// ---------------------------------------------------------------------------
// warp-cooperative reset (csrc/arc_sim.c:88-110, csrc/arc_terrain.c:35-71):
// each lane draws one consecutive slice of the world's RNG stream (skipping
// ahead to it), all lanes build the terrain columns, lane 0 poses the robot.
// The columns' jitter draws go straight into the world's own terrain array,
// each to the slot its height later overwrites, so a warp needs only ~7 KB
// of shared memory and dozens of worlds reset side by side on every SM.

constexpr int kLat1 = (kGridMax / 8 + 2) * (kGridMax / 8 + 2);   // 100
constexpr int kLat2 = (kGridMax / 3 + 2) * (kGridMax / 3 + 2);   // 529

struct ResetSmem {
    double lat[kLat1 + kLat2];
    // lattice coordinates of column index i for the two spacings (8, 3):
    // integer part and smoothed fraction (csrc/arc_terrain.c:41-45)
    double frac[2][kGridMax];
    int whole[2][kGridMax];
    uint32_t pose[kMaxJoints + 1];  // the stance noise and yaw draws
};

// The generator's arithmetic is written with explicitly rounded FP64
// operations (no FMA contraction): the quantisation to 0.03 m steps and the
// base shift must see the reference's roundings bit for bit
// (csrc/arc_terrain.c:84-123 evaluates each operation separately).
__device__ __forceinline__ double smooth(double t)
{
    return __dmul_rn(__dmul_rn(t, t), __dsub_rn(3.0, __dmul_rn(2.0, t)));
}

__device__ __forceinline__ void lattice_coord(int spacing, int i, int& g, double& t)
{
    const double f = __ddiv_rn((double)i, (double)spacing);
    g = (int)f;
    t = smooth(__dsub_rn(f, (double)g));
}

__device__ __forceinline__ double noise_at(const double* lat, int m, const double* frac, const int* whole, int ix,
                                           int iy)
{
    const int gx = whole[ix], gy = whole[iy];
    const double tx = frac[ix], ty = frac[iy];
    double a = lat[gx + gy * m], b = lat[gx + 1 + gy * m];
    double c = lat[gx + (gy + 1) * m], d = lat[gx + 1 + (gy + 1) * m];
    double top = __dadd_rn(a, __dmul_rn(__dsub_rn(b, a), tx));
    double bot = __dadd_rn(c, __dmul_rn(__dsub_rn(d, c), tx));
    return __dadd_rn(__dmul_rn(top, __dsub_rn(1.0, ty)), __dmul_rn(bot, ty));
}

// one column: hills + bumps + jitter, quantised (csrc/arc_terrain.c:93-118)
__device__ __forceinline__ double column_height(const ResetSmem& sm, const double* lat1, int m1, const double* lat2,
                                                int m2, int ix, int iy, double amp1, double amp2, double ampj,
                                                uint32_t draw)
{
    double v = __dadd_rn(0.0, __dmul_rn(amp1, noise_at(lat1, m1, sm.frac[0], sm.whole[0], ix, iy)));
    v = __dadd_rn(v, __dmul_rn(amp2, noise_at(lat2, m2, sm.frac[1], sm.whole[1], ix, iy)));
    const double u = __dmul_rn((double)draw, 1.0 / 4294967296.0);
    const double jitter = __dadd_rn(-1.0, __dmul_rn(2.0, u));
    const double hj = __dadd_rn(v, __dmul_rn(ampj, jitter));
    return __dmul_rn(0.03, floor(__dadd_rn(__ddiv_rn(hj, 0.03), 0.5)));
}

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
__device__ void reset_world_warp(ResetSmem& sm, const ResetModel& RM, const Worlds<R>& W, TerrainGeom<R>* tg,
                                 TerrainGeomD* tgd, int i, uint32_t seed, double diff, int n, double cell)
{
    const int lane = threadIdx.x & 31;
    n = n < kGridMax ? n : kGridMax;
    const bool rough = diff > 0.0;
    const int m1 = n / 8 + 2, m2 = n / 3 + 2;
    const int L = rough ? m1 * m1 + m2 * m2 : 0;
    const int J = rough ? n * n : 0;
    R* h = W.th + W.toff[i];
    if (!terrain_column_ok(W, i, (long long)n * n - 1, kCheckTerrainWrite))
        return;  // the whole warp: n and the slice are the world's
    // the raw jitter draw of column c sits in the low word of h[c] until the
    // column's height replaces it
    uint32_t* hdraw = reinterpret_cast<uint32_t*>(h);
    constexpr int kStep = sizeof(R) / sizeof(uint32_t);
    {
        // slices of 2^kSliceBits draws: a lane skips by its index times a
        // power of two, a few columns of five tables
        constexpr int kSliceBits = 8;
        const int total = L + J + RM.nj + 1;
        const int per = total <= 32 << kSliceBits ? 1 << kSliceBits : (total + 31) / 32;
        const int first = lane * per, last = first + per < total ? first + per : total;
        Xorshift rng;
        rng.seed(seed);
        if (first < last)
            rng_skip(rng, (uint32_t)first);
        for (int k = first; k < last; ++k) {
            const uint32_t u = rng.next();
            if (k < L)
                sm.lat[k] = __dadd_rn(-1.0, __dmul_rn(2.0, __dmul_rn((double)u, 1.0 / 4294967296.0)));
            else if (k < L + J)
                hdraw[(k - L) * kStep] = u;
            else
                sm.pose[k - L - J] = u;
        }
    }
    for (int c = lane; c < 2 * kGridMax; c += 32)
        lattice_coord(c < kGridMax ? 8 : 3, c % kGridMax, sm.whole[c / kGridMax][c % kGridMax],
                      sm.frac[c / kGridMax][c % kGridMax]);
    __syncwarp();

    TerrainGeomD g;
    g.nx = g.ny = n;
    g.cell = cell;
    g.ox = -0.5 * n * cell;
    g.oy = -0.5 * n * cell;
    g.outside = -100.0;
    if (lane == 0) {
        tgd[i] = g;
        tg[i] = TerrainGeom<R>{n, n, (R)g.cell, (R)g.ox, (R)g.oy, (R)g.outside};
    }
    const double reach = RM.footprint + 0.1, step = 0.5 * cell;
    bool out_x = false, out_y = false;
    const unsigned long long mx = scan_cells(reach, step, g.ox, cell, n, out_x);
    const unsigned long long my = scan_cells(reach, step, g.oy, cell, n, out_y);
    double ground = (out_x || out_y) ? g.outside : -1e30;
    if (!rough) {
        for (int c = lane; c < n * n; c += 32)
            h[c] = R(0);
        if (mx && my)
            ground = ground > 0.0 ? ground : 0.0;
    } else {
        const double amp1 = __dmul_rn(0.45, diff), amp2 = __dmul_rn(0.12, diff), ampj = __dmul_rn(0.06, diff);
        const double* lat1 = sm.lat;
        const double* lat2 = sm.lat + m1 * m1;
        const double f0x = floor((0.0 - g.ox) / g.cell), f0y = floor((0.0 - g.oy) / g.cell);
        double base = g.outside;
        if (f0x >= 0.0 && f0y >= 0.0 && f0x < n && f0y < n) {
            const int ix = (int)f0x, iy = (int)f0y;
            base = column_height(sm, lat1, m1, lat2, m2, ix, iy, amp1, amp2, ampj, hdraw[(ix + iy * n) * kStep]);
        }
        __syncwarp();  // every lane has read the base column's draw
        double gmax = -1e300;
        for (int c = lane; c < n * n; c += 32) {
            const int ix = c % n, iy = c / n;
            const double hf =
                __dsub_rn(column_height(sm, lat1, m1, lat2, m2, ix, iy, amp1, amp2, ampj, hdraw[c * kStep]), base);
            h[c] = (R)hf;
            if (((mx >> ix) & 1) && ((my >> iy) & 1))
                gmax = gmax > hf ? gmax : hf;
        }
        for (int off = 16; off > 0; off >>= 1) {
            double o = __shfl_xor_sync(0xffffffffu, gmax, off);
            gmax = gmax > o ? gmax : o;
        }
        if (mx && my)
            ground = ground > gmax ? ground : gmax;
    }
    if (lane != 0)
        return;

    // noisy stance, yaw, forward kinematics (csrc/arc_sim.c:99-109, csrc/arc_phys.c:749-782)
    double angles[kMaxJoints];
    for (int j = 0; j < RM.nj; ++j) {
        double a = RM.default_angles[j] + range_of(sm.pose[j], -0.1, 0.1);
        angles[j] = a < RM.lo[j] ? RM.lo[j] : (a > RM.hi[j] ? RM.hi[j] : a);
    }
    const double yaw = range_of(sm.pose[RM.nj], -kPi, kPi);
    V3<double> xs[kMaxBodies];
    Q4<double> qs[kMaxBodies];
    const double sy = sin(0.5 * yaw), cyw = cos(0.5 * yaw);
    xs[0] = V3<double>{0.0, 0.0, ground + RM.stand_height + 0.03};
    qs[0] = qnormalize(Q4<double>{cyw, 0.0 * sy, 0.0 * sy, 1.0 * sy});
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
__global__ void __launch_bounds__(32)
k_reset_warp(const __grid_constant__ ResetModel RM, Worlds<R> W, TerrainGeom<R>* tg, TerrainGeomD* tgd,
             const int* __restrict__ ids, int n_ids, const unsigned* __restrict__ seeds,
             const double* __restrict__ difficulty, const int* __restrict__ grid_of, double cell)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ResetSmem& sm = *reinterpret_cast<ResetSmem*>(smem_raw);
    for (int k = blockIdx.x; k < n_ids; k += gridDim.x) {
        const int i = ids[k];
        reset_world_warp(sm, RM, W, tg, tgd, i, seeds[k], difficulty[k], grid_of ? grid_of[i] : kGridMax, cell);
        __syncwarp();
    }
}

// ArcTask.reset (arc/task.py:113-125) + the observation of the new episode,
// by the 32 lanes of one warp (compiled once, as task_step_world).
template <class R>
__device__ __noinline__ void task_reset_world(ResetSmem& sm, const DevModel<R>& M, const ResetModel& RM, const Worlds<R>& W,
                                 TerrainGeom<R>* tg, TerrainGeomD* tgd, const int* __restrict__ grid_of, double cell,
                                 const TaskParams& P, const TaskState& S, float* obs, int i)
{
    const int lane = threadIdx.x & 31;
    uint32_t seed = 0;
    if (lane == 0) {
        const unsigned e = S.episode[i]++;
        seed = (uint32_t)stream_u64(P.seed, key_of(S, i), 2u, e);
        S.difficulty[i] = S.level[i];
    }
    seed = __shfl_sync(0xffffffffu, seed, 0);
    __syncwarp();
    reset_world_warp(sm, RM, W, tg, tgd, i, seed, S.difficulty[i], grid_of ? grid_of[i] : kGridMax, cell);
    __syncwarp();
    if (lane == 0) {
        for (int j = 0; j < kNumJoints; ++j)
            S.prev_action[(size_t)i * kNumJoints + j] = 0.0f;
        S.torso_steps[i] = 0;
        S.steps[i] = 0;
        S.checkpoints[i] = 0;
        Obs64 o;
        read_world(M, W, i, o);
        place_target(P, W, S, i, o.x, o.rot);
        if (obs)
            write_obs(P, W, S, i, o, obs + (size_t)i * kObsSize);
    }
    __syncwarp();
}

template <class R>
__global__ void __launch_bounds__(32)
k_task_reset(const __grid_constant__ DevModel<R> M, const __grid_constant__ ResetModel RM, Worlds<R> W,
             TerrainGeom<R>* tg, TerrainGeomD* tgd, const int* __restrict__ grid_of, double cell,
             const __grid_constant__ TaskParams P, TaskState S, float* obs, const int* __restrict__ ids,
             const int* __restrict__ count_dev, int max_n)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ResetSmem& sm = *reinterpret_cast<ResetSmem*>(smem_raw);
    const int n = count_dev ? min(*count_dev, max_n) : max_n;
    for (int k = blockIdx.x; k < n; k += gridDim.x)
        task_reset_world(sm, M, RM, W, tg, tgd, grid_of, cell, P, S, obs, ids[k]);
}

template <class R>
__global__ void k_task_set_targets(Worlds<R> W, const __grid_constant__ TaskParams P, TaskState S,
                                   const int* __restrict__ ids, const double* __restrict__ xy, int n)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    const int i = ids[k];
    const R* rec = W.rec + (size_t)i * W.stride;
    V3<double> pos{(double)rec[0], (double)rec[1], (double)rec[2]};
    Q4<double> q{(double)rec[3], (double)rec[4], (double)rec[5], (double)rec[6]};
    M3<double> rot = m3_from_quat(q);
    const double tx = xy[2 * k], ty = xy[2 * k + 1];
    S.target[2 * i] = tx;
    S.target[2 * i + 1] = ty;
    S.target_z[i] = height_at(W, i, tx, ty);
    const double dx = tx - pos.x, dy = ty - pos.y;
    S.prev_dist[i] = sqrt(dx * dx + dy * dy);
    S.prev_gaze[i] = gaze_error(rot, pos, S.target + 2 * i);
    S.in_view[i] = S.prev_gaze[i] < P.fov_rad;
}

// ---------------------------------------------------------------------------
// The warp-per-leg step (FP32, the quadruped) and, fused with it, the task
// layer of ArcVecEnv.step_wait (arc/env.py:99-117). One kernel template
// serves every form, instantiated per form:
//   kPhysics      the step alone (arc_sim_step, the separate env step, tiles
//                 of substeps);
//   kWithTask     each CTA steps a group of 32 worlds, then, before its next
//                 group, runs the task step on them (warp 0, one lane per
//                 world) and their observations' heights (all threads); the
//                 ended worlds go to the ended-world list, which a separate
//                 reset launch then takes;
//   kWithResets   the same, and the group's ended worlds are reset in the
//                 kernel too, one warp each.
// The task functions are compiled once (not inlined) and called both from
// the fused forms and from the separate task kernels, so their outputs do
// not depend on the form. The physics is inlined into each instantiation:
// the physics-only one then holds no task code, gets the registers it needs
// without spills (126, against 128 and spills when the task code shares the
// kernel) and steps 6 % faster; the fused instantiations compile the same
// physics source in another context and agree with it to FP32 rounding
// rather than bit for bit. The ended-world list is filled in completion
// order, as the separate task kernel fills it.
enum : int { kPhysics = 0, kWithTask = 1, kWithResets = 2 };

struct ControlSmem {
    union {
        wl::Smem step;
        ResetSmem reset[wl::kWarps];  // one per warp, after the group's step
    };
    int ended[wl::kWorlds];  // worlds of the group whose episode ended
    int n_ended;
    int next;  // the next group from the work queue
};

template <int kMode>
__global__ void __launch_bounds__(wl::kThreads, 4)
k_control_step(const __grid_constant__ DevModel<float> M, const __grid_constant__ ResetModel RM, Worlds<float> W,
               TerrainGeom<float>* tg, TerrainGeomD* tgd, const int* __restrict__ grid_of, double cell,
               const __grid_constant__ TaskParams P, TaskState S, TaskOut O, Actuation A,
               float* __restrict__ spill, int spill_per_lane, int lane_cap, const int* __restrict__ ids, int n_items,
               int* queue, int sub0, int sub1, float* __restrict__ tile_q)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ControlSmem& cs = *reinterpret_cast<ControlSmem*>(smem_raw);
    const int tid = threadIdx.x, leg = tid / wl::kWorlds, j = tid % wl::kWorlds;
    const int n_groups = (n_items + wl::kWorlds - 1) / wl::kWorlds;
    auto world_of = [&](int item) {
        const int w = item < n_items ? (ids ? ids[item] : item) : -1;
        return w >= 0 && w < W.n ? w : -1;
    };
    (void)world_of;  // the physics-only form takes no task work
    // with a queue every group, the first included, is taken from it: a CTA
    // that becomes resident only when others leave finds the queue empty
    // instead of holding back a group of its own
    int first = blockIdx.x;
    if (queue) {
        if (tid == 0)
            cs.next = atomicAdd(queue, 1);
        __syncthreads();
        first = cs.next;
    }
#pragma unroll 1
    for (int group = first; group < n_groups;) {
        wl::step_group(cs.step, M, W, A, spill, spill_per_lane, lane_cap, ids, n_items, group, tid, leg, j, sub0, sub1,
                       tile_q);
        if constexpr (kMode != kPhysics) {
            if (tid == 0)
                cs.n_ended = 0;
            __syncthreads();
            // arc/task.py:155-259 but the heights; warp 0's lane j takes the
            // world its own lane stepped as leg 0 (time and unstable written by it)
            if (tid < wl::kWorlds) {
                const int world = world_of(group * wl::kWorlds + j);
                if (world >= 0 && task_step_world(M, W, P, S, O, A.actions32, 2, world))
                    cs.ended[atomicAdd(&cs.n_ended, 1)] = world;
            }
            __syncthreads();
#pragma unroll 1
            for (int t = tid; t < wl::kWorlds * kHeightParts; t += wl::kThreads) {
                const int world = world_of(group * wl::kWorlds + t / kHeightParts);
                if (world >= 0)
                    task_heights_part(W, P, O, world, t % kHeightParts);
            }
            if constexpr (kMode == kWithResets) {
                __syncthreads();
#pragma unroll 1
                for (int e = leg; e < cs.n_ended; e += wl::kWarps)
                    task_reset_world(cs.reset[leg], M, RM, W, tg, tgd, grid_of, cell, P, S, O.obs, cs.ended[e]);
            }
        }
        if (!queue)
            break;
        __syncthreads();  // this group's task and reset work is done with the shared memory
        if (tid == 0)
            cs.next = atomicAdd(queue, 1);
        __syncthreads();
        group = cs.next;
    }
    if (queue) {
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            if (atomicAdd(queue + 1, 1) == (int)gridDim.x - 1) {
                queue[0] = 0;
                queue[1] = 0;
                __threadfence();
            }
        }
    }
}

// One launch of k_control_step<kMode> over the n_items worlds ids[0 .. n_items).
template <int kMode>
cudaError_t launch_form(const DevModel<float>& M, const ResetModel& RM, const Worlds<float>& W,
                        TerrainGeom<float>* tg, TerrainGeomD* tgd, const int* grid_of, double cell,
                        const TaskParams& P, const TaskState& S, const TaskOut& O, const Actuation& A, float* spill,
                        int spill_per_lane, int lane_cap, const int* ids, int n_items, int* queue, int sub0, int sub1,
                        float* tile_q, cudaStream_t stream)
{
    const int smem = (int)sizeof(ControlSmem);
    // per device and form: the shared-memory attribute, and how many CTAs are
    // resident at once (the work queue's wave)
    static std::atomic<unsigned long long> configured{0};
    static int resident[64] = {};
    cudaError_t e = once_per_device(configured, [&](int dev) {
        cudaError_t r = cudaFuncSetAttribute(k_control_step<kMode>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        int sms = 0, per_sm = 0;
        if (r == cudaSuccess)
            r = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (r == cudaSuccess)
            r = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_control_step<kMode>, wl::kThreads, smem);
        if (r == cudaSuccess)
            resident[dev] = sms * (per_sm > 0 ? per_sm : 1);
        return r;
    });
    if (e != cudaSuccess)
        return e;
    const int groups = (n_items + wl::kWorlds - 1) / wl::kWorlds;
    int grid = groups;
    if (queue) {
        int dev = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess)
            return e;
        grid = groups < resident[dev] ? groups : resident[dev];  // one wave of resident CTAs
    }
    k_control_step<kMode><<<grid, wl::kThreads, smem, stream>>>(M, RM, W, tg, tgd, grid_of, cell, P, S, O, A, spill,
                                                                spill_per_lane, lane_cap, ids, n_items, queue, sub0,
                                                                sub1, tile_q);
    return cudaGetLastError();
}

cudaError_t control_launch(const DevModel<float>& M, const ResetModel& RM, const Worlds<float>& W,
                           TerrainGeom<float>* tg, TerrainGeomD* tgd, const int* grid_of, double cell,
                           const TaskParams& P, const TaskState& S, const TaskOut& O, const Actuation& A,
                           float* spill, int spill_per_lane, int lane_cap, const int* ids, int n_items, int* queue,
                           int mode, int sub0, int sub1, float* tile_q, cudaStream_t stream)
{
    switch (mode) {
    case kPhysics:
        return launch_form<kPhysics>(M, RM, W, tg, tgd, grid_of, cell, P, S, O, A, spill, spill_per_lane, lane_cap,
                                     ids, n_items, queue, sub0, sub1, tile_q, stream);
    case kWithTask:
        return launch_form<kWithTask>(M, RM, W, tg, tgd, grid_of, cell, P, S, O, A, spill, spill_per_lane, lane_cap,
                                      ids, n_items, queue, sub0, sub1, tile_q, stream);
    case kWithResets:
        return launch_form<kWithResets>(M, RM, W, tg, tgd, grid_of, cell, P, S, O, A, spill, spill_per_lane,
                                        lane_cap, ids, n_items, queue, sub0, sub1, tile_q, stream);
    default:
        return cudaErrorInvalidValue;
    }
}

template <class R>
__global__ void k_env_admit(TaskState S, const int* __restrict__ ids, const double* __restrict__ difficulty,
                            const unsigned* __restrict__ keys, int n)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    const int i = ids[k];
    S.level[i] = difficulty[k];
    S.difficulty[i] = difficulty[k];
    S.key[i] = keys[k];
    S.episode[i] = 0;
    S.draws[i] = 0;
}

int reset_grid(int n)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int cap = sms * 32;  // one warp per world, up to 32 resident per SM
    return n < cap ? (n > 0 ? n : 1) : cap;
}

}  // namespace

template <class R>
cudaError_t launch_task_step(const DevModel<R>& M, const Worlds<R>& W, const TaskParams& P, const TaskState& S,
                             const TaskOut& O, const float* actions, int write_obs_rows, cudaStream_t stream, int first,
                             int count, const int* ids)
{
    if (count < 0)
        count = W.n - first;
    if (count <= 0 || (!ids && (first < 0 || first + count > W.n)))
        return count == 0 ? cudaSuccess : cudaErrorInvalidValue;
    k_task_step<R><<<(count + 127) / 128, 128, 0, stream>>>(M, W, P, S, O, actions, write_obs_rows, first, count, ids);
    return cudaGetLastError();
}

template <class R>
cudaError_t launch_task_heights(const DevModel<R>& M, const Worlds<R>& W, const TaskParams& P, const TaskOut& O,
                                cudaStream_t stream, int first, int count, const int* ids)
{
    if (count < 0)
        count = W.n - first;
    if (count <= 0 || (!ids && (first < 0 || first + count > W.n)))
        return count == 0 ? cudaSuccess : cudaErrorInvalidValue;
    const long long threads = (long long)count * kHeightParts;
    k_task_heights<R><<<(unsigned)((threads + kHeightThreads - 1) / kHeightThreads), kHeightThreads, 0, stream>>>(
        M, W, P, O, first, count, ids);
    return cudaGetLastError();
}

template <class R>
cudaError_t launch_task_observe(const DevModel<R>& M, const Worlds<R>& W, const TaskParams& P, const TaskState& S,
                                float* obs, const int* ids, int n_ids, cudaStream_t stream)
{
    if (n_ids <= 0)
        return cudaSuccess;
    k_task_observe<R><<<(n_ids + 127) / 128, 128, 0, stream>>>(M, W, P, S, obs, ids, n_ids);
    return cudaGetLastError();
}

template <class R>
cudaError_t launch_task_reset(const DevModel<R>& M, const ResetModel& RM, const Worlds<R>& W, TerrainGeom<R>* tg,
                              TerrainGeomD* tgd, const int* grid_of, double cell, const TaskParams& P,
                              const TaskState& S, float* obs, const int* ids, const int* count_dev, int max_n,
                              cudaStream_t stream)
{
    if (max_n <= 0)
        return cudaSuccess;
    static std::atomic<unsigned long long> configured{0};
    cudaError_t e = once_per_device(configured, [](int) {
        return cudaFuncSetAttribute(k_task_reset<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(ResetSmem));
    });
    if (e != cudaSuccess)
        return e;
    k_task_reset<R><<<reset_grid(max_n), 32, sizeof(ResetSmem), stream>>>(M, RM, W, tg, tgd, grid_of, cell, P, S, obs,
                                                                       ids, count_dev, max_n);
    return cudaGetLastError();
}

template <class R>
cudaError_t launch_task_set_targets(const Worlds<R>& W, const TaskParams& P, const TaskState& S, const int* ids,
                                    const double* xy, int n, cudaStream_t stream)
{
    if (n <= 0)
        return cudaSuccess;
    k_task_set_targets<R><<<(n + 127) / 128, 128, 0, stream>>>(W, P, S, ids, xy, n);
    return cudaGetLastError();
}

cudaError_t init_reset_tables(cudaStream_t stream)
{
    k_jump_init<<<kJumpBits, 128, 0, stream>>>();
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? cudaStreamSynchronize(stream) : e;
}

template <class R>
cudaError_t launch_reset_warp(const ResetModel& RM, const Worlds<R>& W, TerrainGeom<R>* tg, TerrainGeomD* tgd,
                              const int* ids, int n_ids, const unsigned* seeds, const double* difficulty,
                              const int* grid_of, double cell, cudaStream_t stream)
{
    if (n_ids <= 0)
        return cudaSuccess;
    static std::atomic<unsigned long long> configured{0};
    cudaError_t e = once_per_device(configured, [](int) {
        return cudaFuncSetAttribute(k_reset_warp<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(ResetSmem));
    });
    if (e != cudaSuccess)
        return e;
    k_reset_warp<R><<<reset_grid(n_ids), 32, sizeof(ResetSmem), stream>>>(RM, W, tg, tgd, ids, n_ids, seeds,
                                                                        difficulty, grid_of, cell);
    return cudaGetLastError();
}

template <class R>
cudaError_t launch_env_admit(const DevModel<R>& M, const ResetModel& RM, const Worlds<R>& W, TerrainGeom<R>* tg,
                             TerrainGeomD* tgd, const int* grid_of, double cell, const TaskParams& P,
                             const TaskState& S, float* obs, const int* ids, const double* difficulty,
                             const unsigned* keys, int n, cudaStream_t stream)
{
    if (n <= 0)
        return cudaSuccess;
    if (!S.key)
        return cudaErrorInvalidValue;
    k_env_admit<R><<<(n + 127) / 128, 128, 0, stream>>>(S, ids, difficulty, keys, n);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return e;
    return launch_task_reset<R>(M, RM, W, tg, tgd, grid_of, cell, P, S, obs, ids, nullptr, n, stream);
}

cudaError_t launch_control_step(const DevModel<float>& M, const ResetModel& RM, const Worlds<float>& W,
                                TerrainGeom<float>* tg, TerrainGeomD* tgd, const int* grid_of, double cell,
                                const TaskParams& P, const TaskState& S, const TaskOut& O, const float* actions,
                                float* spill, int spill_per_lane, int lane_cap, const int* ids, int n_items, int* queue,
                                bool resets, cudaStream_t stream)
{
    if (W.n <= 0 || n_items <= 0)
        return cudaSuccess;
    if (!M.leaper)
        return cudaErrorInvalidValue;
    return control_launch(M, RM, W, tg, tgd, grid_of, cell, P, S, O, Actuation{nullptr, actions}, spill,
                          spill_per_lane, lane_cap, ids, n_items, queue, resets ? kWithResets : kWithTask, 0,
                          M.substeps, nullptr, stream);
}

cudaError_t launch_step_warps(const DevModel<float>& M, const Worlds<float>& W, const Actuation& A, float* spill,
                              int spill_per_lane, int lane_cap, const int* ids, int n_items, int* queue,
                              cudaStream_t stream, int tile, float* tile_q)
{
    if (W.n <= 0 || n_items <= 0)
        return cudaSuccess;
    if (!M.leaper)
        return cudaErrorInvalidValue;
    // the task layer's parameters, which the physics alone does not read
    static const ResetModel RM{};
    static const TaskParams P{};
    if (tile <= 0 || tile >= M.substeps || !tile_q)
        tile = M.substeps;
    for (int sub0 = 0; sub0 < M.substeps; sub0 += tile) {
        const int sub1 = sub0 + tile < M.substeps ? sub0 + tile : M.substeps;
        cudaError_t e = control_launch(M, RM, W, nullptr, nullptr, nullptr, 0.0, P, TaskState{}, TaskOut{}, A, spill,
                                       spill_per_lane, lane_cap, ids, n_items, queue, kPhysics, sub0, sub1, tile_q,
                                       stream);
        if (e != cudaSuccess)
            return e;
    }
    return cudaSuccess;
}

#define ARC_INSTANTIATE_TASK(R)                                                                                    \
    template cudaError_t launch_task_step<R>(const DevModel<R>&, const Worlds<R>&, const TaskParams&,            \
                                             const TaskState&, const TaskOut&, const float*, int, cudaStream_t,  \
                                             int, int, const int*);                                              \
    template cudaError_t launch_task_heights<R>(const DevModel<R>&, const Worlds<R>&, const TaskParams&,         \
                                                const TaskOut&, cudaStream_t, int, int, const int*);             \
    template cudaError_t launch_task_observe<R>(const DevModel<R>&, const Worlds<R>&, const TaskParams&,         \
                                                const TaskState&, float*, const int*, int, cudaStream_t);        \
    template cudaError_t launch_task_reset<R>(const DevModel<R>&, const ResetModel&, const Worlds<R>&,           \
                                              TerrainGeom<R>*, TerrainGeomD*, const int*, double,                \
                                              const TaskParams&, const TaskState&, float*, const int*,           \
                                              const int*, int, cudaStream_t);                                    \
    template cudaError_t launch_task_set_targets<R>(const Worlds<R>&, const TaskParams&, const TaskState&,       \
                                                    const int*, const double*, int, cudaStream_t);               \
    template cudaError_t launch_env_admit<R>(const DevModel<R>&, const ResetModel&, const Worlds<R>&,            \
                                             TerrainGeom<R>*, TerrainGeomD*, const int*, double, const TaskParams&, \
                                             const TaskState&, float*, const int*, const double*, const unsigned*, \
                                             int, cudaStream_t);                                                  \
    template cudaError_t launch_reset_warp<R>(const ResetModel&, const Worlds<R>&, TerrainGeom<R>*,              \
                                              TerrainGeomD*, const int*, int, const unsigned*, const double*,    \
                                              const int*, double, cudaStream_t);

ARC_INSTANTIATE_TASK(float)
ARC_INSTANTIATE_TASK(double)

}  // namespace arc
