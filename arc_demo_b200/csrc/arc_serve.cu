// arc_serve.cu - a serving engine over one batch of resident worlds.
//
// No counterpart in the reference, which steps one synchronous batch per
// call (arc/env.py:96-117). Clients submit requests - n worlds (fresh
// episodes: seeds, difficulties) to be stepped k control steps with given
// actions, or with actions from a seeded Ornstein-Uhlenbeck process - and
// wait for the worlds' final states. One engine thread runs continuous
// batching over a fixed pool of world slots (the byte budget, decided at
// create):
//   - admission: queued requests are admitted first come, first served,
//     while free slots hold them; their slots are reset (arc_sim_reset) at
//     once;
//   - one tick: every admitted request's worlds step together in one launch
//     (arc_sim_step_ids over the active slot list), whatever request they
//     belong to;
//   - eviction: a request whose k steps are done has its final states read
//     back and its slots freed at the end of that tick.
// A world's result depends only on its own state and actions (worlds never
// interact, and the step runs the same per-world code for any slot list),
// so a request's results in the mix equal its results alone, bit for bit.
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
constexpr int kReadChunk = 16384;  // worlds per read-back of final states
// an observation row: root 13, rotation 9, joints 36, contacts 6, flag 1
// (the blocks of arc_sim_observe, csrc/arc_sim.h:17-21)
constexpr int kObsRow = 13 + 9 + 36 + 6 + 1;

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

// Actions of the listed slots for this tick: the request's own (host
// actions, uploaded compactly beside the list) or the next value of the
// slot's OU process, theta = 0.15, sigma = 0.3, clipped to [-1, 1].
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

// New requests' slots: OU state zero, step count zero, the per-world seed.
__global__ void k_admit(const int* __restrict__ ids, const unsigned long long* __restrict__ seeds, int n,
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

using Clock = std::chrono::steady_clock;

struct Request {
    long long id = 0;
    int n = 0, steps = 0, done_steps = 0;
    std::vector<unsigned> seeds;
    std::vector<double> difficulty;
    std::vector<float> actions;  // steps x n x 12, or empty: OU
    unsigned long long ou_seed = 0;
    std::vector<int> slots;
    double* user_out = nullptr;  // the caller's result buffer, or NULL
    std::vector<double> out;     // the result when the caller gave none
    double* dest() { return user_out ? user_out : out.data(); }
    Clock::time_point t_submit, t_admit, t_done;
    bool done = false;
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
    int capacity = 0, state_size = 0, device = 0;
    int result = ARC_SERVE_STATE, row = 0;  // doubles per world in a result
    std::vector<int> free_slots;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Request>> queue;
    std::vector<std::shared_ptr<Request>> active;  // engine thread only
    std::unordered_map<long long, std::shared_ptr<Request>> by_id;
    long long next_id = 0;
    bool stop = false;
    std::thread engine;
    cudaStream_t stream = nullptr;
    // device and pinned staging, capacity-sized
    DevArray<int> d_ids, d_admit_ids;
    DevArray<float> d_actions, d_ou, d_given;
    DevArray<int> d_t;
    DevArray<unsigned long long> d_seed, d_admit_seeds;
    DevArray<unsigned char> d_use;
    HostArray<int> h_ids, h_admit_ids;
    HostArray<float> h_given;
    HostArray<unsigned char> h_use;
    HostArray<unsigned long long> h_admit_seeds;
    HostArray<double> h_state;  // kReadChunk final states or observation blocks, pinned
    HostArray<int> h_read_ids, h_flags;
    DevArray<int> d_read_ids, d_flags;
    DevArray<double> d_obs;     // root, rot, joints, contacts blocks of kReadChunk rows
    // statistics (under mu)
    long long ticks = 0, world_steps = 0, completed = 0;
    int max_active = 0;
    double busy_s = 0.0, admit_s = 0.0, step_s = 0.0, evict_s = 0.0;
    int error = 0;
};

namespace {

bool ok(cudaError_t e, arc_server* sv, const char* what)
{
    if (e == cudaSuccess)
        return true;
    std::fprintf(stderr, "arc_server: %s: %s\n", what, cudaGetErrorString(e));
    return false;
}

// Admits queued requests in order while they fit; resets their worlds.
bool admit(arc_server* sv)
{
    std::vector<std::shared_ptr<Request>> admitted;
    {
        std::lock_guard<std::mutex> lock(sv->mu);
        while (!sv->queue.empty() && (int)sv->free_slots.size() >= sv->queue.front()->n) {
            auto r = sv->queue.front();
            sv->queue.pop_front();
            r->slots.assign(sv->free_slots.end() - r->n, sv->free_slots.end());
            sv->free_slots.resize(sv->free_slots.size() - r->n);
            r->t_admit = Clock::now();
            admitted.push_back(r);
        }
    }
    if (admitted.empty())
        return true;
    int m = 0;
    std::vector<int> ids;
    std::vector<unsigned> seeds;
    std::vector<double> diff;
    for (auto& r : admitted) {
        for (int i = 0; i < r->n; ++i) {
            sv->h_admit_ids.p[m] = r->slots[i];
            // one OU stream per (request, world)
            sv->h_admit_seeds.p[m] = r->ou_seed * 0x9e3779b97f4a7c15ull + (unsigned long long)i;
            ++m;
        }
        ids.insert(ids.end(), r->slots.begin(), r->slots.end());
        seeds.insert(seeds.end(), r->seeds.begin(), r->seeds.end());
        diff.insert(diff.end(), r->difficulty.begin(), r->difficulty.end());
        sv->active.push_back(r);
    }
    arc_sim_reset(sv->sim, ids.data(), (int)ids.size(), seeds.data(), diff.data());
    if (arc_sim_last_error(sv->sim))
        return false;
    if (!ok(cudaMemcpyAsync(sv->d_admit_ids.p, sv->h_admit_ids.p, sizeof(int) * m, cudaMemcpyHostToDevice,
                            sv->stream), sv, "admit ids") ||
        !ok(cudaMemcpyAsync(sv->d_admit_seeds.p, sv->h_admit_seeds.p, sizeof(unsigned long long) * m,
                            cudaMemcpyHostToDevice, sv->stream), sv, "admit seeds"))
        return false;
    k_admit<<<(m + 127) / 128, 128, 0, sv->stream>>>(sv->d_admit_ids.p, sv->d_admit_seeds.p, m, sv->d_seed.p,
                                                     sv->d_ou.p, sv->d_t.p);
    return ok(cudaGetLastError(), sv, "admit kernel");
}

// One control step of every active world; completes finished requests.
bool tick(arc_server* sv)
{
    const auto t0 = Clock::now();
    int n = 0;
    bool any_given = false;
    for (auto& r : sv->active) {
        const bool given = !r->actions.empty();
        any_given |= given;
        for (int i = 0; i < r->n; ++i, ++n) {
            sv->h_ids.p[n] = r->slots[i];
            sv->h_use.p[n] = given;
            if (given)
                std::memcpy(sv->h_given.p + (size_t)n * kJ,
                            r->actions.data() + ((size_t)r->done_steps * r->n + i) * kJ, sizeof(float) * kJ);
        }
    }
    if (n == 0)
        return true;
    cudaStream_t st = sv->stream;
    if (!ok(cudaMemcpyAsync(sv->d_ids.p, sv->h_ids.p, sizeof(int) * n, cudaMemcpyHostToDevice, st), sv, "ids") ||
        !ok(cudaMemcpyAsync(sv->d_use.p, sv->h_use.p, n, cudaMemcpyHostToDevice, st), sv, "flags"))
        return false;
    if (any_given &&
        !ok(cudaMemcpyAsync(sv->d_given.p, sv->h_given.p, sizeof(float) * kJ * n, cudaMemcpyHostToDevice, st), sv,
            "actions"))
        return false;
    k_tick_actions<<<(n + 127) / 128, 128, 0, st>>>(sv->d_ids.p, n, sv->d_given.p, sv->d_use.p, sv->d_seed.p,
                                                    sv->d_ou.p, sv->d_t.p, sv->d_actions.p);
    if (!ok(cudaGetLastError(), sv, "action kernel"))
        return false;
    if (arc_sim_step_ids(sv->sim, sv->d_ids.p, n, nullptr, sv->d_actions.p, st) != ARC_OK)
        return false;
    if (!ok(cudaStreamSynchronize(st), sv, "tick"))
        return false;
    const auto t1 = Clock::now();
    // evict finished requests
    std::vector<std::shared_ptr<Request>> keep, finished;
    for (auto& r : sv->active)
        (++r->done_steps >= r->steps ? finished : keep).push_back(r);
    // results of every finished request, in pinned chunks
    const size_t row_n = (size_t)sv->row;
    for (auto& r : finished)
        if (!r->user_out)
            r->out.resize((size_t)r->n * row_n);
    size_t total = 0;
    for (auto& r : finished)
        total += r->n;
    std::vector<std::pair<Request*, int>> owners;  // (request, world index) of each row of the chunk
    size_t row = 0, ri = 0, wi = 0;
    while (row < total) {
        const int m = (int)std::min<size_t>(kReadChunk, total - row);
        owners.resize(m);
        for (int k = 0; k < m; ++k) {
            Request* r = finished[ri].get();
            sv->h_read_ids.p[k] = r->slots[wi];
            owners[k] = {r, (int)wi};
            if (++wi == (size_t)r->n) {
                wi = 0;
                ++ri;
            }
        }
        int rc = ARC_OK;
        if (sv->result == ARC_SERVE_STATE) {
            rc = arc_sim_get_state(sv->sim, sv->h_read_ids.p, m, sv->h_state.p);
        } else {
            double* d = sv->d_obs.p;
            double *d_root = d, *d_rot = d + (size_t)m * 13, *d_j = d_rot + (size_t)m * 9,
                   *d_c = d_j + (size_t)m * 36;
            rc = (ok(cudaMemcpyAsync(sv->d_read_ids.p, sv->h_read_ids.p, sizeof(int) * m, cudaMemcpyHostToDevice,
                                     sv->stream), sv, "read ids")
                      ? arc_sim_observe_ids(sv->sim, sv->d_read_ids.p, m, d_root, d_rot, d_j, d_c, sv->d_flags.p,
                                            sv->stream)
                      : ARC_ERR_CUDA);
            if (rc == ARC_OK &&
                !(ok(cudaMemcpyAsync(sv->h_state.p, d, sizeof(double) * (size_t)m * (kObsRow - 1),
                                     cudaMemcpyDeviceToHost, sv->stream), sv, "observations") &&
                  ok(cudaMemcpyAsync(sv->h_flags.p, sv->d_flags.p, sizeof(int) * m, cudaMemcpyDeviceToHost,
                                     sv->stream), sv, "flags") &&
                  ok(cudaStreamSynchronize(sv->stream), sv, "read back")))
                rc = ARC_ERR_CUDA;
        }
        for (int k = 0; k < m; ++k) {
            Request* r = owners[k].first;
            double* dst = r->dest() + (size_t)owners[k].second * row_n;
            if (rc) {
                r->status = rc;
            } else if (sv->result == ARC_SERVE_STATE) {
                std::memcpy(dst, sv->h_state.p + (size_t)k * row_n, sizeof(double) * row_n);
            } else {
                const double* h = sv->h_state.p;
                std::memcpy(dst, h + (size_t)k * 13, sizeof(double) * 13);
                std::memcpy(dst + 13, h + (size_t)m * 13 + (size_t)k * 9, sizeof(double) * 9);
                std::memcpy(dst + 22, h + (size_t)m * 22 + (size_t)k * 36, sizeof(double) * 36);
                std::memcpy(dst + 58, h + (size_t)m * 58 + (size_t)k * 6, sizeof(double) * 6);
                dst[64] = (double)sv->h_flags.p[k];
            }
        }
        row += m;
    }
    sv->active.swap(keep);
    std::lock_guard<std::mutex> lock(sv->mu);
    sv->step_s += std::chrono::duration<double>(t1 - t0).count();
    sv->evict_s += std::chrono::duration<double>(Clock::now() - t1).count();
    ++sv->ticks;
    sv->world_steps += n;
    sv->max_active = std::max(sv->max_active, n);
    if (!finished.empty()) {
        const auto now = Clock::now();
        for (auto& r : finished) {
            sv->free_slots.insert(sv->free_slots.end(), r->slots.begin(), r->slots.end());
            r->t_done = now;
            r->done = true;
            ++sv->completed;
        }
        sv->cv_done.notify_all();
    }
    return true;
}

void engine_loop(arc_server* sv)
{
    cudaSetDevice(sv->device);
    for (;;) {
        {
            std::unique_lock<std::mutex> lock(sv->mu);
            sv->cv_work.wait(lock, [&] { return sv->stop || !sv->queue.empty() || !sv->active.empty(); });
            if (sv->stop)
                return;
        }
        const auto t0 = Clock::now();
        bool good = admit(sv);
        {
            std::lock_guard<std::mutex> lock(sv->mu);
            sv->admit_s += std::chrono::duration<double>(Clock::now() - t0).count();
        }
        good = good && tick(sv);
        std::lock_guard<std::mutex> lock(sv->mu);
        sv->busy_s += std::chrono::duration<double>(Clock::now() - t0).count();
        if (!good) {
            // fail everything outstanding; the engine stops stepping
            sv->error = ARC_ERR_CUDA;
            for (auto& r : sv->active) {
                r->status = sv->error;
                r->done = true;
            }
            sv->active.clear();
            for (auto& r : sv->queue) {
                r->status = sv->error;
                r->done = true;
            }
            sv->queue.clear();
            sv->cv_done.notify_all();
            sv->stop = true;
            return;
        }
    }
}

}  // namespace

extern "C" arc_server* arc_server_create(int capacity, double dt, int substeps, int grid, double cell, int result)
{
    if (capacity <= 0 || (result != ARC_SERVE_STATE && result != ARC_SERVE_OBSERVE))
        return nullptr;
    auto* sv = new arc_server();
    cudaGetDevice(&sv->device);
    sv->sim = arc_sim_create(capacity, dt, substeps, grid, cell);
    if (!sv->sim) {
        delete sv;
        return nullptr;
    }
    sv->capacity = capacity;
    sv->state_size = arc_sim_state_size(sv->sim);
    sv->result = result;
    sv->row = result == ARC_SERVE_STATE ? sv->state_size : kObsRow;
    const size_t chunk = (size_t)std::min(capacity, kReadChunk);
    arc_sim_set_kernel(sv->sim, ARC_KERNEL_WARPS, 32);
    sv->stream = static_cast<cudaStream_t>(arc_sim_stream(sv->sim));
    const size_t c = (size_t)capacity;
    const bool good = cudaMalloc(&sv->d_ids.p, c * sizeof(int)) == cudaSuccess &&
                      cudaMalloc(&sv->d_admit_ids.p, c * sizeof(int)) == cudaSuccess &&
                      cudaMalloc(&sv->d_actions.p, c * kJ * sizeof(float)) == cudaSuccess &&
                      cudaMalloc(&sv->d_ou.p, c * kJ * sizeof(float)) == cudaSuccess &&
                      cudaMalloc(&sv->d_given.p, c * kJ * sizeof(float)) == cudaSuccess &&
                      cudaMalloc(&sv->d_t.p, c * sizeof(int)) == cudaSuccess &&
                      cudaMalloc(&sv->d_seed.p, c * sizeof(unsigned long long)) == cudaSuccess &&
                      cudaMalloc(&sv->d_admit_seeds.p, c * sizeof(unsigned long long)) == cudaSuccess &&
                      cudaMalloc(&sv->d_use.p, c) == cudaSuccess &&
                      cudaMallocHost(&sv->h_ids.p, c * sizeof(int)) == cudaSuccess &&
                      cudaMallocHost(&sv->h_admit_ids.p, c * sizeof(int)) == cudaSuccess &&
                      cudaMallocHost(&sv->h_given.p, c * kJ * sizeof(float)) == cudaSuccess &&
                      cudaMallocHost(&sv->h_use.p, c) == cudaSuccess &&
                      cudaMallocHost(&sv->h_admit_seeds.p, c * sizeof(unsigned long long)) == cudaSuccess &&
                      cudaMallocHost(&sv->h_state.p, chunk * sv->row * sizeof(double)) == cudaSuccess &&
                      cudaMallocHost(&sv->h_read_ids.p, chunk * sizeof(int)) == cudaSuccess &&
                      cudaMallocHost(&sv->h_flags.p, chunk * sizeof(int)) == cudaSuccess &&
                      cudaMalloc(&sv->d_read_ids.p, chunk * sizeof(int)) == cudaSuccess &&
                      cudaMalloc(&sv->d_flags.p, chunk * sizeof(int)) == cudaSuccess &&
                      cudaMalloc(&sv->d_obs.p, chunk * (kObsRow - 1) * sizeof(double)) == cudaSuccess;
    if (!good) {
        std::fprintf(stderr, "arc_server_create: allocation failed for %d slots\n", capacity);
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
            r->done = true;
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

extern "C" long long arc_server_submit(arc_server* sv, int n_worlds, int n_steps, const unsigned* seeds,
                                       const double* difficulty, const float* actions, unsigned long long ou_seed,
                                       double* out)
{
    if (!sv || n_worlds <= 0 || n_worlds > sv->capacity || n_steps <= 0 || !seeds || !difficulty)
        return ARC_ERR_ARG;
    auto r = std::make_shared<Request>();
    r->n = n_worlds;
    r->steps = n_steps;
    r->seeds.assign(seeds, seeds + n_worlds);
    r->difficulty.assign(difficulty, difficulty + n_worlds);
    if (actions)
        r->actions.assign(actions, actions + (size_t)n_steps * n_worlds * kJ);
    r->ou_seed = ou_seed;
    r->user_out = out;
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lock(sv->mu);
        if (sv->stop)
            return sv->error ? sv->error : ARC_ERR_ARG;
        r->id = sv->next_id++;
        sv->by_id[r->id] = r;
        sv->queue.push_back(r);
    }
    sv->cv_work.notify_one();
    return r->id;
}

extern "C" int arc_server_wait(arc_server* sv, long long id, double timeout_s, double* out, double* times)
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
        if (!sv->cv_done.wait_until(lock, until, [&] { return r->done; }))
            return 0;
        sv->by_id.erase(id);
    }
    if (r->status)
        return r->status;
    if (out && !r->user_out)
        std::memcpy(out, r->out.data(), sizeof(double) * r->out.size());
    if (times) {
        times[0] = std::chrono::duration<double>(r->t_admit - r->t_submit).count();
        times[1] = std::chrono::duration<double>(r->t_done - r->t_admit).count();
        times[2] = std::chrono::duration<double>(r->t_done - r->t_submit).count();
    }
    return 1;
}

extern "C" int arc_server_stats(arc_server* sv, double* stats)
{
    if (!sv || !stats)
        return ARC_ERR_ARG;
    std::lock_guard<std::mutex> lock(sv->mu);
    stats[0] = (double)sv->ticks;
    stats[1] = (double)sv->world_steps;
    stats[2] = sv->busy_s;
    stats[3] = (double)sv->max_active;
    stats[4] = (double)sv->completed;
    stats[5] = (double)sv->queue.size();
    stats[6] = sv->admit_s;
    stats[7] = sv->step_s;
    stats[8] = sv->evict_s;
    return sv->error;
}
