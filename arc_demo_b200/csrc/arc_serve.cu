// arc_serve.cu - a serving engine: client sessions of resident worlds with the
// task layer, stepped by continuous batching.
//
// No counterpart in the reference, whose ArcVecEnv steps one synchronous batch
// per call (arc/env.py:96-117). Here:
//   - a session is one client's batch of n worlds with the task layer
//     (ArcTask: observations, rewards, terminations, auto-reset). Opening it
//     queues it for n slots of a fixed pool of worlds (the device-memory
//     budget, decided at create). Once slots are free it is admitted: each
//     world starts an episode at the session's difficulty, its random streams
//     named by the session's key (arc_env_admit), so the session's worlds
//     behave alike whichever slots they get. The session keeps its slots, and
//     its worlds stay on the device, until it is closed.
//   - a request steps one session's worlds k control steps, with given
//     actions or a seeded Ornstein-Uhlenbeck process, and returns every
//     step's rewards and done flags and the observations after the last
//     step. A world whose episode ends (terminated or truncated,
//     arc/task.py:196-220) is evicted from its slot at once and the slot
//     reset with the world's next episode, as ArcVecEnv auto-resets
//     (arc/env.py:99-117).
//   - one engine thread runs continuous batching: each tick steps the worlds
//     of every running request together (arc_env_step_ids: one launch of the
//     fused control step over their slots), whatever session they belong to.
//     A queued request starts running, first come first served, once its
//     session is resident, runs no other request, and the tick has room for
//     its worlds: at most tick_cap worlds run at once, so a burst of large
//     requests lengthens the queue, not every tick; a request larger than
//     the cap runs alone. It leaves the tick when its k steps are done.
// Worlds never interact and the fused step runs the same per-world code for
// any list of slots, so a session's results in the mix equal its results
// alone, bit for bit.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/arc_sim.h"

namespace {

constexpr int kJ = 12;
constexpr int kObs = 195;           // arc/task.py:231-259
constexpr int kReadChunk = 16384;   // worlds per read-back of final observations

// Counter-based normal draws for the OU actions: splitmix64 of (seed, count)
// gives two uniforms, Box-Muller gives the normal.
__device__ __forceinline__ unsigned long long mix64(unsigned long long z)
{
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ float normal_draw(unsigned long long seed, unsigned long long k)
{
    const unsigned long long a = mix64(seed ^ mix64(2 * k)), b = mix64(seed ^ mix64(2 * k + 1));
    const float u1 = ((float)(a >> 40) + 1.0f) * (1.0f / 16777216.0f);  // (0, 1]
    const float u2 = (float)(b >> 40) * (1.0f / 16777216.0f);
    return sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
}

// Actions of the listed slots for this tick into the env's action rows: the
// request's own (host actions, uploaded compactly beside the list) or the
// next value of the slot's OU process, theta = 0.15, sigma = 0.3, clipped to
// [-1, 1].
__global__ void k_tick_actions(const int* __restrict__ ids, int n, const float* __restrict__ given,
                               const unsigned char* __restrict__ use_given, const unsigned long long* __restrict__ seed,
                               float* __restrict__ ou, int* __restrict__ t, float* __restrict__ actions)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    const int s = ids[k];
    if (use_given[k]) {
        for (int c = 0; c < kJ; ++c)
            actions[(size_t)s * kJ + c] = given[(size_t)k * kJ + c];
        return;
    }
    const int step = t[s];
    for (int c = 0; c < kJ; ++c) {
        float x = ou[(size_t)s * kJ + c];
        x += 0.15f * (0.0f - x) + 0.3f * normal_draw(seed[s], (unsigned long long)step * kJ + c);
        ou[(size_t)s * kJ + c] = x;
        actions[(size_t)s * kJ + c] = fminf(fmaxf(x, -1.0f), 1.0f);
    }
    t[s] = step + 1;
}

// A starting request's slots: OU state zero, step count zero, the per-world seed.
__global__ void k_start(const int* __restrict__ ids, const unsigned long long* __restrict__ seeds, int n,
                        unsigned long long* __restrict__ seed, float* __restrict__ ou, int* __restrict__ t)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    const int s = ids[k];
    seed[s] = seeds[k];
    t[s] = 0;
    for (int c = 0; c < kJ; ++c)
        ou[(size_t)s * kJ + c] = 0.0f;
}

// The tick's rewards and done flags (bit 0 terminated, bit 1 truncated), in
// tick order.
__global__ void k_gather_step(const int* __restrict__ ids, int n, const float* __restrict__ reward,
                              const unsigned char* __restrict__ terminated, const unsigned char* __restrict__ truncated,
                              float* __restrict__ out_reward, unsigned char* __restrict__ out_done)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    const int s = ids[k];
    out_reward[k] = reward[s];
    out_done[k] = (unsigned char)((terminated[s] ? 1 : 0) | (truncated[s] ? 2 : 0));
}

// Observation rows of the listed slots, in list order.
__global__ void k_gather_obs(const int* __restrict__ ids, int n, const float* __restrict__ obs, float* __restrict__ out)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * kObs)
        return;
    const int k = (int)(t / kObs), c = (int)(t % kObs);
    out[t] = obs[(size_t)ids[k] * kObs + c];
}

using Clock = std::chrono::steady_clock;

struct Session {
    long long id = 0;
    int n = 0;
    unsigned long long key = 0;
    std::vector<double> difficulty;
    std::vector<int> slots;
    bool admitted = false, closed = false, busy = false;
    int pending = 0;  // requests submitted and not finished
};

struct Request {
    long long id = 0;
    std::shared_ptr<Session> ses;
    int steps = 0, done_steps = 0;
    std::vector<float> actions;  // steps x n x 12, or empty: OU
    unsigned long long ou_seed = 0;
    float* obs = nullptr;            // n x 195, or NULL
    float* reward = nullptr;         // steps x n, or NULL
    unsigned char* done = nullptr;   // steps x n, or NULL
    Clock::time_point t_submit, t_start, t_done;
    bool finished = false;
    int status = 0;
};

template <class T> struct DevArray {
    T* p = nullptr;
    ~DevArray() { cudaFree(p); }
};
template <class T> struct HostArray {
    T* p = nullptr;
    ~HostArray() { cudaFreeHost(p); }
};

}  // namespace

struct arc_server {
    arc_sim* sim = nullptr;
    int capacity = 0, tick_cap = 0, device = 0;
    std::vector<int> free_slots;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::unordered_map<long long, std::shared_ptr<Session>> sessions;
    std::deque<std::shared_ptr<Session>> waiting;      // sessions waiting for slots
    std::deque<std::shared_ptr<Request>> queue;        // requests not running yet
    std::vector<std::shared_ptr<Request>> running;     // engine thread only
    std::unordered_map<long long, std::shared_ptr<Request>> by_id;
    long long next_id = 1;
    bool stop = false;
    std::thread engine;
    cudaStream_t stream = nullptr;
    // the env's device buffers (rows indexed by slot)
    float *env_actions = nullptr, *env_obs = nullptr, *env_reward = nullptr;
    unsigned char *env_terminated = nullptr, *env_truncated = nullptr;
    // per-slot OU state and per-tick staging, capacity-sized
    DevArray<int> d_ids, d_start_ids;
    DevArray<float> d_ou, d_given, d_reward, d_obs;
    DevArray<int> d_t;
    DevArray<unsigned long long> d_seed, d_start_seeds;
    DevArray<unsigned char> d_use, d_done;
    HostArray<int> h_ids, h_start_ids;
    HostArray<float> h_given, h_reward, h_obs;
    HostArray<unsigned char> h_use, h_done;
    HostArray<unsigned long long> h_start_seeds;
    // statistics (under mu)
    long long ticks = 0, world_steps = 0, completed = 0, episodes_ended = 0;
    int max_active = 0;
    double busy_s = 0.0, admit_s = 0.0, step_s = 0.0, read_s = 0.0;
    int error = 0;
};

namespace {

bool ok(cudaError_t e, const char* what)
{
    if (e == cudaSuccess)
        return true;
    std::fprintf(stderr, "arc_server: %s: %s\n", what, cudaGetErrorString(e));
    return false;
}

// A world's key: its session's key and its index in the session.
unsigned world_key(unsigned long long session_key, int i)
{
    unsigned long long z = session_key * 0x9e3779b97f4a7c15ull + (unsigned long long)i + 1;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return (unsigned)((z ^ (z >> 31)) & 0x7fffffffu);
}

// Admits waiting sessions in order while free slots hold them; frees the
// slots of closed sessions with nothing left to run.
bool admit(arc_server* sv)
{
    std::vector<std::shared_ptr<Session>> admitted;
    {
        std::lock_guard<std::mutex> lock(sv->mu);
        for (auto it = sv->sessions.begin(); it != sv->sessions.end();) {
            Session& s = *it->second;
            if (s.closed && s.pending == 0) {
                if (s.admitted)
                    sv->free_slots.insert(sv->free_slots.end(), s.slots.begin(), s.slots.end());
                it = sv->sessions.erase(it);
            } else {
                ++it;
            }
        }
        while (!sv->waiting.empty() && (int)sv->free_slots.size() >= sv->waiting.front()->n) {
            auto s = sv->waiting.front();
            sv->waiting.pop_front();
            if (s->closed && s->pending == 0)
                continue;  // closed before admission with nothing to run (a closed session's queued requests still run)
            s->slots.assign(sv->free_slots.end() - s->n, sv->free_slots.end());
            sv->free_slots.resize(sv->free_slots.size() - s->n);
            admitted.push_back(s);
        }
    }
    for (auto& s : admitted) {
        std::vector<unsigned> keys(s->n);
        for (int i = 0; i < s->n; ++i)
            keys[i] = world_key(s->key, i);
        if (arc_env_admit(sv->sim, s->slots.data(), s->n, s->difficulty.data(), keys.data(), sv->stream) != ARC_OK)
            return false;
        std::lock_guard<std::mutex> lock(sv->mu);
        s->admitted = true;
    }
    return true;
}

// Starts queued requests, first come first served, whose session is
// resident and idle, while the tick has room.
bool start(arc_server* sv)
{
    std::vector<std::shared_ptr<Request>> started;
    {
        std::lock_guard<std::mutex> lock(sv->mu);
        int active = 0;
        for (auto& r : sv->running)
            active += r->ses->n;
        for (auto it = sv->queue.begin(); it != sv->queue.end();) {
            Request& r = **it;
            if (!r.ses->admitted || r.ses->busy) {
                ++it;
                continue;
            }
            if (active > 0 && active + r.ses->n > sv->tick_cap)
                break;  // the oldest runnable request waits for room; none overtakes it
            r.ses->busy = true;
            r.t_start = Clock::now();
            active += r.ses->n;
            started.push_back(*it);
            it = sv->queue.erase(it);
        }
    }
    if (started.empty())
        return true;
    int m = 0;
    for (auto& r : started)
        for (int i = 0; i < r->ses->n; ++i, ++m) {
            sv->h_start_ids.p[m] = r->ses->slots[i];
            // one OU stream per (request, world)
            sv->h_start_seeds.p[m] = r->ou_seed * 0x9e3779b97f4a7c15ull + (unsigned long long)i;
        }
    if (!ok(cudaMemcpyAsync(sv->d_start_ids.p, sv->h_start_ids.p, sizeof(int) * m, cudaMemcpyHostToDevice, sv->stream),
            "start ids") ||
        !ok(cudaMemcpyAsync(sv->d_start_seeds.p, sv->h_start_seeds.p, sizeof(unsigned long long) * m,
                            cudaMemcpyHostToDevice, sv->stream),
            "start seeds"))
        return false;
    k_start<<<(m + 127) / 128, 128, 0, sv->stream>>>(sv->d_start_ids.p, sv->d_start_seeds.p, m, sv->d_seed.p,
                                                     sv->d_ou.p, sv->d_t.p);
    if (!ok(cudaGetLastError(), "start kernel"))
        return false;
    sv->running.insert(sv->running.end(), started.begin(), started.end());
    return true;
}

// Reads back the final observations of finished requests, in pinned chunks.
bool read_obs(arc_server* sv, const std::vector<std::shared_ptr<Request>>& finished)
{
    std::vector<std::pair<Request*, int>> owners;
    size_t ri = 0;
    int wi = 0;
    while (ri < finished.size()) {
        int m = 0;
        owners.clear();
        while (ri < finished.size() && m < kReadChunk) {
            Request* r = finished[ri].get();
            if (!r->obs) {
                ++ri;
                continue;
            }
            sv->h_ids.p[m] = r->ses->slots[wi];
            owners.push_back({r, wi});
            ++m;
            if (++wi == r->ses->n) {
                wi = 0;
                ++ri;
            }
        }
        if (m == 0)
            break;
        if (!ok(cudaMemcpyAsync(sv->d_ids.p, sv->h_ids.p, sizeof(int) * m, cudaMemcpyHostToDevice, sv->stream),
                "obs ids"))
            return false;
        const long long total = (long long)m * kObs;
        k_gather_obs<<<(unsigned)((total + 255) / 256), 256, 0, sv->stream>>>(sv->d_ids.p, m, sv->env_obs,
                                                                              sv->d_obs.p);
        if (!ok(cudaGetLastError(), "obs gather") ||
            !ok(cudaMemcpyAsync(sv->h_obs.p, sv->d_obs.p, sizeof(float) * total, cudaMemcpyDeviceToHost, sv->stream),
                "obs copy") ||
            !ok(cudaStreamSynchronize(sv->stream), "obs read-back"))
            return false;
        for (int k = 0; k < m; ++k)
            std::memcpy(owners[k].first->obs + (size_t)owners[k].second * kObs, sv->h_obs.p + (size_t)k * kObs,
                        sizeof(float) * kObs);
    }
    return true;
}

// One control step of every running request's worlds; completes finished requests.
bool tick(arc_server* sv)
{
    const auto t0 = Clock::now();
    int n = 0;
    bool any_given = false;
    for (auto& r : sv->running) {
        const bool given = !r->actions.empty();
        any_given |= given;
        const int rn = r->ses->n;
        for (int i = 0; i < rn; ++i, ++n) {
            sv->h_ids.p[n] = r->ses->slots[i];
            sv->h_use.p[n] = given;
            if (given)
                std::memcpy(sv->h_given.p + (size_t)n * kJ,
                            r->actions.data() + ((size_t)r->done_steps * rn + i) * kJ, sizeof(float) * kJ);
        }
    }
    if (n == 0)
        return true;
    cudaStream_t st = sv->stream;
    if (!ok(cudaMemcpyAsync(sv->d_ids.p, sv->h_ids.p, sizeof(int) * n, cudaMemcpyHostToDevice, st), "ids") ||
        !ok(cudaMemcpyAsync(sv->d_use.p, sv->h_use.p, n, cudaMemcpyHostToDevice, st), "flags"))
        return false;
    if (any_given &&
        !ok(cudaMemcpyAsync(sv->d_given.p, sv->h_given.p, sizeof(float) * kJ * n, cudaMemcpyHostToDevice, st),
            "actions"))
        return false;
    k_tick_actions<<<(n + 127) / 128, 128, 0, st>>>(sv->d_ids.p, n, sv->d_given.p, sv->d_use.p, sv->d_seed.p,
                                                    sv->d_ou.p, sv->d_t.p, sv->env_actions);
    if (!ok(cudaGetLastError(), "action kernel"))
        return false;
    if (arc_env_step_ids(sv->sim, sv->d_ids.p, n, st) != ARC_OK)
        return false;
    k_gather_step<<<(n + 127) / 128, 128, 0, st>>>(sv->d_ids.p, n, sv->env_reward, sv->env_terminated,
                                                   sv->env_truncated, sv->d_reward.p, sv->d_done.p);
    if (!ok(cudaGetLastError(), "gather kernel") ||
        !ok(cudaMemcpyAsync(sv->h_reward.p, sv->d_reward.p, sizeof(float) * n, cudaMemcpyDeviceToHost, st),
            "rewards") ||
        !ok(cudaMemcpyAsync(sv->h_done.p, sv->d_done.p, n, cudaMemcpyDeviceToHost, st), "done flags") ||
        !ok(cudaStreamSynchronize(st), "tick"))
        return false;
    const auto t1 = Clock::now();
    std::vector<std::shared_ptr<Request>> keep, finished;
    long long ended = 0;
    int off = 0;
    for (auto& r : sv->running) {
        const int rn = r->ses->n;
        const size_t at = (size_t)r->done_steps * rn;
        if (r->reward)
            std::memcpy(r->reward + at, sv->h_reward.p + off, sizeof(float) * rn);
        if (r->done)
            std::memcpy(r->done + at, sv->h_done.p + off, rn);
        for (int i = 0; i < rn; ++i)
            ended += sv->h_done.p[off + i] != 0;
        off += rn;
        (++r->done_steps >= r->steps ? finished : keep).push_back(r);
    }
    const bool read = read_obs(sv, finished);
    sv->running.swap(keep);
    std::lock_guard<std::mutex> lock(sv->mu);
    sv->step_s += std::chrono::duration<double>(t1 - t0).count();
    sv->read_s += std::chrono::duration<double>(Clock::now() - t1).count();
    ++sv->ticks;
    sv->world_steps += n;
    sv->episodes_ended += ended;
    sv->max_active = std::max(sv->max_active, n);
    if (!finished.empty()) {
        const auto now = Clock::now();
        for (auto& r : finished) {
            r->t_done = now;
            r->status = read ? 0 : ARC_ERR_CUDA;
            r->finished = true;
            r->ses->busy = false;
            --r->ses->pending;
            ++sv->completed;
        }
        sv->cv_done.notify_all();
    }
    return read;
}

bool has_work(arc_server* sv)
{
    if (sv->stop || !sv->running.empty())
        return true;
    for (auto& r : sv->queue)
        if (r->ses->admitted && !r->ses->busy)
            return true;
    if (!sv->waiting.empty() && (int)sv->free_slots.size() >= sv->waiting.front()->n)
        return true;
    for (auto& kv : sv->sessions)
        if (kv.second->closed && kv.second->pending == 0)
            return true;
    return false;
}

void fail_all(arc_server* sv, int status)
{
    for (auto& r : sv->running) {
        r->status = status;
        r->finished = true;
    }
    sv->running.clear();
    for (auto& r : sv->queue) {
        r->status = status;
        r->finished = true;
    }
    sv->queue.clear();
    sv->cv_done.notify_all();
}

void engine_loop(arc_server* sv)
{
    cudaSetDevice(sv->device);
    for (;;) {
        {
            std::unique_lock<std::mutex> lock(sv->mu);
            sv->cv_work.wait(lock, [&] { return has_work(sv); });
            if (sv->stop)
                return;
        }
        const auto t0 = Clock::now();
        bool good = admit(sv);
        const auto t1 = Clock::now();
        good = good && start(sv) && tick(sv);
        std::lock_guard<std::mutex> lock(sv->mu);
        sv->admit_s += std::chrono::duration<double>(t1 - t0).count();
        sv->busy_s += std::chrono::duration<double>(Clock::now() - t0).count();
        if (!good) {
            // fail everything outstanding; the engine stops stepping
            sv->error = ARC_ERR_CUDA;
            fail_all(sv, sv->error);
            sv->stop = true;
            return;
        }
    }
}

}  // namespace

extern "C" arc_server* arc_server_create(int capacity, double dt, int substeps, int grid, double cell,
                                         const arc_task_config* cfg, int tick_cap)
{
    if (capacity <= 0 || tick_cap < 0)
        return nullptr;
    auto* sv = new arc_server();
    cudaGetDevice(&sv->device);
    sv->sim = arc_sim_create(capacity, dt, substeps, grid, cell);
    if (!sv->sim) {
        delete sv;
        return nullptr;
    }
    arc_task_config c;
    if (cfg) {
        c = *cfg;
    } else {
        arc_task_config_default(&c);
        c.curriculum = 0;  // each session's worlds keep the difficulty it asked for
    }
    c.dt = dt;
    sv->capacity = capacity;
    sv->tick_cap = tick_cap > 0 ? tick_cap : capacity;
    arc_sim_set_kernel(sv->sim, ARC_KERNEL_WARPS, 32);
    arc_sim_set_work_queue(sv->sim, 1);
    sv->stream = static_cast<cudaStream_t>(arc_sim_stream(sv->sim));
    void* p = nullptr;
    bool good = arc_env_init(sv->sim, &c, 0x5eedull) == ARC_OK;
    auto buffer = [&](int which) {
        p = nullptr;
        good = good && arc_env_buffer(sv->sim, which, &p, nullptr, nullptr, nullptr, nullptr) == ARC_OK;
        return p;
    };
    sv->env_actions = static_cast<float*>(buffer(ARC_ENV_ACTIONS));
    sv->env_obs = static_cast<float*>(buffer(ARC_ENV_OBS));
    sv->env_reward = static_cast<float*>(buffer(ARC_ENV_REWARD));
    sv->env_terminated = static_cast<unsigned char*>(buffer(ARC_ENV_TERMINATED));
    sv->env_truncated = static_cast<unsigned char*>(buffer(ARC_ENV_TRUNCATED));
    const size_t n = (size_t)capacity, chunk = (size_t)std::min(capacity, kReadChunk);
    good = good && cudaMalloc(&sv->d_ids.p, n * sizeof(int)) == cudaSuccess &&
           cudaMalloc(&sv->d_start_ids.p, n * sizeof(int)) == cudaSuccess &&
           cudaMalloc(&sv->d_ou.p, n * kJ * sizeof(float)) == cudaSuccess &&
           cudaMalloc(&sv->d_given.p, n * kJ * sizeof(float)) == cudaSuccess &&
           cudaMalloc(&sv->d_reward.p, n * sizeof(float)) == cudaSuccess &&
           cudaMalloc(&sv->d_obs.p, chunk * kObs * sizeof(float)) == cudaSuccess &&
           cudaMalloc(&sv->d_t.p, n * sizeof(int)) == cudaSuccess &&
           cudaMalloc(&sv->d_seed.p, n * sizeof(unsigned long long)) == cudaSuccess &&
           cudaMalloc(&sv->d_start_seeds.p, n * sizeof(unsigned long long)) == cudaSuccess &&
           cudaMalloc(&sv->d_use.p, n) == cudaSuccess && cudaMalloc(&sv->d_done.p, n) == cudaSuccess &&
           cudaMallocHost(&sv->h_ids.p, n * sizeof(int)) == cudaSuccess &&
           cudaMallocHost(&sv->h_start_ids.p, n * sizeof(int)) == cudaSuccess &&
           cudaMallocHost(&sv->h_given.p, n * kJ * sizeof(float)) == cudaSuccess &&
           cudaMallocHost(&sv->h_reward.p, n * sizeof(float)) == cudaSuccess &&
           cudaMallocHost(&sv->h_obs.p, chunk * kObs * sizeof(float)) == cudaSuccess &&
           cudaMallocHost(&sv->h_use.p, n) == cudaSuccess && cudaMallocHost(&sv->h_done.p, n) == cudaSuccess &&
           cudaMallocHost(&sv->h_start_seeds.p, n * sizeof(unsigned long long)) == cudaSuccess;
    if (!good) {
        std::fprintf(stderr, "arc_server_create: set-up failed for %d slots\n", capacity);
        arc_sim_destroy(sv->sim);
        delete sv;
        return nullptr;
    }
    sv->free_slots.resize(capacity);
    for (int i = 0; i < capacity; ++i)
        sv->free_slots[i] = capacity - 1 - i;  // slot 0 is handed out first
    sv->engine = std::thread(engine_loop, sv);
    return sv;
}

extern "C" void arc_server_destroy(arc_server* sv)
{
    if (!sv)
        return;
    {
        std::lock_guard<std::mutex> lock(sv->mu);
        sv->stop = true;
        for (auto& r : sv->queue) {
            r->status = ARC_ERR_ARG;
            r->finished = true;
        }
        sv->queue.clear();
        sv->cv_done.notify_all();
    }
    sv->cv_work.notify_all();
    if (sv->engine.joinable())
        sv->engine.join();
    arc_sim_destroy(sv->sim);
    delete sv;
}

extern "C" long long arc_server_open(arc_server* sv, int n_worlds, const double* difficulty, unsigned long long key)
{
    if (!sv || n_worlds <= 0 || !difficulty)
        return ARC_ERR_ARG;
    auto s = std::make_shared<Session>();
    s->n = n_worlds;
    s->key = key;
    s->difficulty.assign(difficulty, difficulty + n_worlds);
    {
        std::lock_guard<std::mutex> lock(sv->mu);
        if (sv->stop)
            return sv->error ? sv->error : ARC_ERR_ARG;
        if (n_worlds > sv->capacity)
            return ARC_ERR_ARG;
        s->id = sv->next_id++;
        sv->sessions[s->id] = s;
        sv->waiting.push_back(s);
    }
    sv->cv_work.notify_one();
    return s->id;
}

extern "C" long long arc_server_request(arc_server* sv, long long session, int n_steps, const float* actions,
                                        unsigned long long ou_seed, float* obs, float* reward, unsigned char* done)
{
    if (!sv || n_steps <= 0)
        return ARC_ERR_ARG;
    auto r = std::make_shared<Request>();
    r->steps = n_steps;
    r->ou_seed = ou_seed;
    r->obs = obs;
    r->reward = reward;
    r->done = done;
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lock(sv->mu);
        if (sv->stop)
            return sv->error ? sv->error : ARC_ERR_ARG;
        auto it = sv->sessions.find(session);
        if (it == sv->sessions.end() || it->second->closed)
            return ARC_ERR_ARG;
        r->ses = it->second;
        if (actions)
            r->actions.assign(actions, actions + (size_t)n_steps * r->ses->n * kJ);
        ++r->ses->pending;
        r->id = sv->next_id++;
        sv->by_id[r->id] = r;
        sv->queue.push_back(r);
    }
    sv->cv_work.notify_one();
    return r->id;
}

extern "C" int arc_server_wait(arc_server* sv, long long id, double timeout_s, double* times)
{
    if (!sv)
        return ARC_ERR_ARG;
    std::shared_ptr<Request> r;
    {
        std::unique_lock<std::mutex> lock(sv->mu);
        auto it = sv->by_id.find(id);
        if (it == sv->by_id.end())
            return ARC_ERR_ARG;
        r = it->second;
        const auto until = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                              std::chrono::duration<double>(std::max(timeout_s, 0.0)));
        if (!sv->cv_done.wait_until(lock, until, [&] { return r->finished; }))
            return 0;
        sv->by_id.erase(id);
    }
    if (r->status)
        return r->status;
    if (times) {
        times[0] = std::chrono::duration<double>(r->t_start - r->t_submit).count();
        times[1] = std::chrono::duration<double>(r->t_done - r->t_start).count();
        times[2] = std::chrono::duration<double>(r->t_done - r->t_submit).count();
    }
    return 1;
}

extern "C" int arc_server_close(arc_server* sv, long long session)
{
    if (!sv)
        return ARC_ERR_ARG;
    {
        std::lock_guard<std::mutex> lock(sv->mu);
        auto it = sv->sessions.find(session);
        if (it == sv->sessions.end() || it->second->closed)
            return ARC_ERR_ARG;
        it->second->closed = true;
    }
    sv->cv_work.notify_one();
    return ARC_OK;
}

extern "C" int arc_server_stats(arc_server* sv, double* stats)
{
    if (!sv || !stats)
        return ARC_ERR_ARG;
    std::lock_guard<std::mutex> lock(sv->mu);
    int resident = 0;
    for (auto& kv : sv->sessions)
        resident += kv.second->admitted ? kv.second->n : 0;
    stats[0] = (double)sv->ticks;
    stats[1] = (double)sv->world_steps;
    stats[2] = sv->busy_s;
    stats[3] = (double)sv->max_active;
    stats[4] = (double)sv->completed;
    stats[5] = (double)sv->queue.size();
    stats[6] = sv->admit_s;
    stats[7] = sv->step_s;
    stats[8] = sv->read_s;
    stats[9] = (double)sv->episodes_ended;
    stats[10] = (double)resident;
    stats[11] = (double)sv->waiting.size();
    return sv->error;
}
