// arc_sim.cu - host runtime behind the C ABI of include/arc_sim.h.
//
// An arc_sim owns one CUDA stream and all device memory of its worlds
// (layout in arc_device.cuh). The reference-compatible calls stage the
// caller's host buffers through device buffers and synchronise before
// returning, like the reference's synchronous OpenMP calls
// (csrc/arc_sim.c:112-215). Errors never cross the ABI as exceptions: the
// void calls record them (arc_sim_last_error) and print them once to stderr.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "arc_model.h"
#include "arc_task.cuh"
#include "../../include/arc_sim.h"

using namespace arc;

struct arc_model {
    ModelHost m;
};

namespace {

struct DevBuffer {
    void* p = nullptr;
    size_t cap = 0;
};

}  // namespace

struct arc_sim {
    int n = 0, substeps = 0, grid = 0, threads = 1;
    double dt = 0.0, cell = 0.0;
    bool fp64 = false;
    int kernel = ARC_KERNEL_LEGS, wpc = 16;
    ModelHost model;
    DevModel<float> mf;
    DevModel<double> md;
    ResetModel rm;
    cudaStream_t stream = nullptr;
    // device state
    void* rec = nullptr;
    int stride = 0, off_sphere = 0, off_joint = 0;
    uint32_t* sph = nullptr;
    int* unstable = nullptr;
    double* time = nullptr;
    void* th = nullptr;
    long long* toff = nullptr;
    void* tg = nullptr;
    TerrainGeomD* tgd = nullptr;
    int* grid_of = nullptr;
    std::vector<int> grid_host;  // terrain capacity of each world: grid_host[i]^2 columns
    size_t th_count = 0;         // columns in the terrain pool
    int* queue = nullptr;        // work queue of the warp-per-leg kernel (two ints)
    bool use_queue = false;
    int fused = 0;  // env control step: 0 separate kernels, 1 fused step and task, 2 and resets (arc_env_set_fused)
    int step_order = 1;  // env step: 0 index order, 1 each range by difficulty band (arc_env_set_step_order)
    void* lastc = nullptr;     // [n][kMaxContacts][kContactRec] R: the last substep's contacts (recording on)
    int* lastn = nullptr;      // [n] their counts
    int substep_tile = 0;      // warp-per-leg step: substeps per launch (0: the whole control step)
    float* tile_q = nullptr;   // [n][13][4] position-pass quaternions between tiles
    void* spill = nullptr;
    int spill_per_lane = 0, lane_cap = 0;
    double spill_cell = 0.0;
    // staging
    DevBuffer st_in, st_in2, st_in3, st_out;
    // page-locked staging of large device-to-host copies (copy_out)
    void* pin[2] = {nullptr, nullptr};
    cudaEvent_t pin_ev[2] = {nullptr, nullptr};
    std::vector<char> skip;  // observe's outputs the caller did not ask for
    std::vector<double> host_tmp;
    arc_world* hworld = nullptr;
    // task layer (arc_env_*)
    bool env = false;
    TaskParams tp;
    TaskState ts{};
    TaskOut to{};
    float* actions = nullptr;
    std::vector<void*> env_allocs;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    cudaStream_t graph_stream = nullptr;
    int graph_kernel = -1, graph_wpc = -1, graph_queue = -1, graph_fused = -1, graph_tile = -1,
        graph_order = -1;  // the captured form
    void* graph_lastc = nullptr;
    // arc_env_step_host: world indices 0..n-1, per-chunk ended-world lists and
    // counts, the two copy streams and their events
    int* iota = nullptr;
    int* order = nullptr;         // the step kernels' world order (k_order_count, k_order_place)
    int* order_counts = nullptr;  // [chunks][bands] worlds per band of each chunk of the order kernels
    int* chunk_done = nullptr;
    int* chunk_count = nullptr;
    int* part_queue = nullptr;  // arc_env_step_part: a work queue (two ints) per part
    cudaStream_t copy_in = nullptr, copy_out = nullptr;
    cudaEvent_t ev[2 * 16 + 2] = {};
    mutable int err = 0;
    mutable std::string msg;
    mutable bool reported = false;
};

namespace {

int real_size(const arc_sim* s) { return s->fp64 ? 8 : 4; }

int fail(const arc_sim* s, int code, const std::string& what)
{
    s->err = code;
    s->msg = what;
    if (!s->reported) {
        std::fprintf(stderr, "arcsim: %s\n", what.c_str());
        s->reported = true;
    }
    return code;
}

int check(const arc_sim* s, cudaError_t e, const char* where)
{
    if (e == cudaSuccess)
        return ARC_OK;
    return fail(s, ARC_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

void* grow(const arc_sim* sc, DevBuffer& b, size_t bytes)
{
    arc_sim* s = const_cast<arc_sim*>(sc);
    if (bytes <= b.cap && b.p)
        return b.p;
    if (b.p)
        cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
    size_t cap = std::max<size_t>(bytes, 256);
    if (check(s, cudaMalloc(&b.p, cap), "cudaMalloc(staging)") != ARC_OK)
        return nullptr;
    b.cap = cap;
    return b.p;
}

#ifdef ARC_DEVICE_CHECKS
}  // namespace
namespace arc {
// the readers of every translation unit's check record (arc_checks.cuh)
std::vector<int (*)(unsigned long long*, bool)>& device_check_readers()
{
    static std::vector<int (*)(unsigned long long*, bool)> readers;
    return readers;
}
int register_device_checks(int (*read)(unsigned long long* record, bool clear))
{
    device_check_readers().push_back(read);
    return 1;
}
}  // namespace arc
namespace {
#endif

template <class R> Worlds<R> view(const arc_sim* s)
{
    Worlds<R> w;
    w.rec = static_cast<R*>(s->rec);
    w.stride = s->stride;
    w.off_sphere = s->off_sphere;
    w.off_joint = s->off_joint;
    w.sph = s->sph;
    w.unstable = s->unstable;
    w.time = s->time;
    w.th = static_cast<R*>(s->th);
    w.toff = s->toff;
    w.tg = static_cast<const TerrainGeom<R>*>(s->tg);
    w.tgd = s->tgd;
    w.n = s->n;
    w.lastc = static_cast<R*>(s->lastc);
    w.lastn = s->lastn;
#ifdef ARC_DEVICE_CHECKS
    w.grid_of = s->grid_of;
#endif
    return w;
}

void rebuild_models(arc_sim* s)
{
    s->model.leaper = is_leaper_topology(s->model);
    s->mf = make_dev_model<float>(s->model, s->dt, s->substeps, 0.6);
    s->md = make_dev_model<double>(s->model, s->dt, s->substeps, 0.6);
    s->rm = make_reset_model(s->model);
}

int ensure_spill(arc_sim* s, double cell)
{
    if (s->spill && cell >= s->spill_cell)
        return ARC_OK;
    const int cap = lane_contact_bound(s->model, cell);
    const int per = std::max(cap - kMinOnChipContacts, 1);
    const size_t bytes = (size_t)std::max(s->n, 1) * 4 * per * 8 * real_size(s);
    void* p = nullptr;
    if (check(s, cudaMalloc(&p, bytes), "cudaMalloc(contact spill)") != ARC_OK)
        return ARC_ERR_CUDA;
    if (s->spill)
        cudaFree(s->spill);
    s->spill = p;
    s->spill_per_lane = per;
    s->lane_cap = std::max(cap, 0);
    s->spill_cell = cell;
    return ARC_OK;
}

template <class R> void template_record(const arc_sim* s, std::vector<R>& rec)
{
    const ModelHost& m = s->model;
    rec.assign(s->stride, R(0));
    for (int b = 0; b < m.nb; ++b) {
        R* r = rec.data() + b * kBodyRec;
        r[0] = (R)m.b[b].x.x; r[1] = (R)m.b[b].x.y; r[2] = (R)m.b[b].x.z;
        r[3] = (R)m.b[b].q.w; r[4] = (R)m.b[b].q.x; r[5] = (R)m.b[b].q.y; r[6] = (R)m.b[b].q.z;
    }
    for (int j = 0; j < m.nj; ++j) {
        R* r = rec.data() + s->off_joint + j * kJointRec;
        r[0] = (R)m.default_angles[j];  // the template's pose sets targets and angles
        r[1] = (R)m.default_angles[j];
    }
}

template <class R> int init_worlds(arc_sim* s)
{
    const int n = s->n, g = s->grid;
    std::vector<R> one;
    template_record<R>(s, one);
    std::vector<R> all((size_t)n * s->stride);
    for (int i = 0; i < n; ++i)
        std::memcpy(all.data() + (size_t)i * s->stride, one.data(), sizeof(R) * s->stride);
    if (check(s, cudaMemcpy(s->rec, all.data(), sizeof(R) * all.size(), cudaMemcpyHostToDevice), "init records"))
        return ARC_ERR_CUDA;
    // flat terrain, outside at the same height (csrc/arc_sim.c:37: template terrain)
    // the pool packs each world's grid_host[i]^2 columns
    std::vector<long long> toff(n);
    std::vector<TerrainGeom<R>> tg(n);
    std::vector<TerrainGeomD> tgd(n);
    const std::vector<int>& grid_of = s->grid_host;
    long long off = 0;
    for (int i = 0; i < n; ++i) {
        const int gi = grid_of[i];
        toff[i] = off;
        off += (long long)gi * gi;
        const TerrainGeomD gd{gi, gi, s->cell, -0.5 * gi * s->cell, -0.5 * gi * s->cell, 0.0};
        tgd[i] = gd;
        tg[i] = TerrainGeom<R>{gi, gi, (R)gd.cell, (R)gd.ox, (R)gd.oy, (R)gd.outside};
    }
    (void)g;
    int rc = ARC_OK;
    rc |= check(s, cudaMemcpy(s->toff, toff.data(), sizeof(long long) * n, cudaMemcpyHostToDevice), "init toff");
    rc |= check(s, cudaMemcpy(s->tg, tg.data(), sizeof(TerrainGeom<R>) * n, cudaMemcpyHostToDevice), "init tg");
    rc |= check(s, cudaMemcpy(s->tgd, tgd.data(), sizeof(TerrainGeomD) * n, cudaMemcpyHostToDevice), "init tgd");
    rc |= check(s, cudaMemcpy(s->grid_of, grid_of.data(), sizeof(int) * n, cudaMemcpyHostToDevice), "init grid");
    rc |= check(s, cudaMemset(s->th, 0, sizeof(R) * s->th_count), "init terrain");
    rc |= check(s, cudaMemset(s->queue, 0, 2 * sizeof(int)), "init queue");
    rc |= check(s, cudaMemset(s->sph, 0, sizeof(uint32_t) * (size_t)n * std::max(s->model.ns, 1)), "init spheres");
    rc |= check(s, cudaMemset(s->unstable, 0, sizeof(int) * n), "init flags");
    rc |= check(s, cudaMemset(s->time, 0, sizeof(double) * n), "init time");
    // the zeroing runs on the legacy default stream, which the sim's
    // non-blocking stream does not wait for: finish it before any kernel
    rc |= check(s, cudaDeviceSynchronize(), "init");
    return rc ? ARC_ERR_CUDA : ARC_OK;
}

void free_all(arc_sim* s)
{
    if (s->graph_exec)
        cudaGraphExecDestroy(s->graph_exec);
    if (s->graph)
        cudaGraphDestroy(s->graph);
    for (void* p : s->env_allocs)
        cudaFree(p);
    void* ps[] = {s->rec, s->sph, s->unstable, s->time, s->th, s->toff, s->tg, s->tgd, s->grid_of, s->spill, s->queue,
                  s->st_in.p, s->st_in2.p, s->st_in3.p, s->st_out.p, s->iota, s->order, s->order_counts, s->chunk_done, s->chunk_count,
                  s->part_queue, s->tile_q, s->lastc, s->lastn};
    for (void* p : ps)
        if (p)
            cudaFree(p);
    for (cudaEvent_t e : s->ev)
        if (e)
            cudaEventDestroy(e);
    for (int k = 0; k < 2; ++k) {
        if (s->pin[k])
            cudaFreeHost(s->pin[k]);
        if (s->pin_ev[k])
            cudaEventDestroy(s->pin_ev[k]);
    }
    for (cudaStream_t c : {s->copy_in, s->copy_out, s->graph_stream})
        if (c)
            cudaStreamDestroy(c);
    if (s->stream)
        cudaStreamDestroy(s->stream);
    delete s->hworld;
}

// the reset kernels' skip table, built once on each device that creates a sim
int ensure_reset_tables(arc_sim* s)
{
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    if (check(s, cudaGetDevice(&dev), "cudaGetDevice"))
        return ARC_ERR_CUDA;
    if (dev < 0 || dev >= 64)
        return fail(s, ARC_ERR_UNSUPPORTED, "more than 64 devices");
    std::lock_guard<std::mutex> lock(mu);
    if (!done[dev]) {
        if (check(s, init_reset_tables(s->stream), "reset tables"))
            return ARC_ERR_CUDA;
        done[dev] = true;
    }
    return ARC_OK;
}

arc_sim* create_with_model(const ModelHost& model, int n, double dt, int substeps, int grid, double cell,
                           unsigned flags, const int* grids = nullptr)
{
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
        std::fprintf(stderr, "arcsim: no CUDA device available\n");
        return nullptr;
    }
    if (n < 0 || substeps <= 0 || !(cell > 0.0))
        return nullptr;
    arc_sim* s = new arc_sim();
    s->n = n;
    s->dt = dt;
    s->substeps = substeps;
    s->grid = std::max(1, std::min(grid, kGridMax));
    s->cell = cell;
    s->grid_host.assign((size_t)std::max(n, 0), s->grid);
    if (grids)
        for (int i = 0; i < n; ++i)
            s->grid_host[i] = grids[i];
    for (int g : s->grid_host)
        s->th_count += (size_t)g * g;
    s->fp64 = (flags & ARC_SIM_FP64) != 0;
    s->model = model;
    rebuild_models(s);
    // the fastest form that steps the model: warp-per-leg (the quadruped, in
    // FP32 or FP64), plain (any model)
    s->kernel = (flags & ARC_SIM_PLAIN) || !s->model.leaper ? ARC_KERNEL_PLAIN : ARC_KERNEL_WARPS;
    const int rs = real_size(s);
    s->off_sphere = s->model.nb * kBodyRec;
    s->off_joint = s->off_sphere + s->model.ns * kSphereRec;
    const int per16 = 16 / rs;
    s->stride = (s->off_joint + s->model.nj * kJointRec + per16 - 1) / per16 * per16;
    // FP32: the eight worlds of a warp stage their records at distinct
    // shared-memory banks when the stride is 4, 12, 20 or 28 mod 32 words
    if (rs == 4)
        while (s->stride % 8 != 4)
            s->stride += 4;
    const size_t nn = (size_t)std::max(n, 1);
    bool ok = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && cudaMalloc(&s->rec, nn * s->stride * rs) == cudaSuccess;
    ok = ok && cudaMalloc((void**)&s->sph, nn * std::max(s->model.ns, 1) * sizeof(uint32_t)) == cudaSuccess;
    ok = ok && cudaMalloc((void**)&s->unstable, nn * sizeof(int)) == cudaSuccess;
    ok = ok && cudaMalloc((void**)&s->time, nn * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc(&s->th, std::max<size_t>(s->th_count, 1) * rs) == cudaSuccess;
    ok = ok && cudaMalloc((void**)&s->queue, 2 * sizeof(int)) == cudaSuccess;
    ok = ok && cudaMalloc((void**)&s->toff, nn * sizeof(long long)) == cudaSuccess;
    ok = ok && cudaMalloc(&s->tg, nn * (s->fp64 ? sizeof(TerrainGeom<double>) : sizeof(TerrainGeom<float>))) ==
                   cudaSuccess;
    ok = ok && cudaMalloc((void**)&s->tgd, nn * sizeof(TerrainGeomD)) == cudaSuccess;
    ok = ok && cudaMalloc((void**)&s->grid_of, nn * sizeof(int)) == cudaSuccess;
    ok = ok && ensure_spill(s, cell) == ARC_OK;
    ok = ok && ensure_reset_tables(s) == ARC_OK;
    if (ok && n > 0)
        ok = (s->fp64 ? init_worlds<double>(s) : init_worlds<float>(s)) == ARC_OK;
    if (!ok) {
        std::fprintf(stderr, "arcsim: device allocation or initialisation failed for %d worlds\n", n);
        free_all(s);
        delete s;
        cudaGetLastError();
        return nullptr;
    }
    return s;
}

bool ids_ok(const arc_sim* s, const int* ids, int n_ids)
{
    for (int k = 0; k < n_ids; ++k)
        if (ids[k] < 0 || ids[k] >= s->n)
            return false;
    return true;
}

int sync(const arc_sim* s, const char* where) { return check(s, cudaStreamSynchronize(s->stream), where); }

// Host memcpy split over a few persistent threads and the caller: copying
// from page-locked staging into the caller's (pageable) arrays is the slow
// half of a large device-to-host transfer. One job at a time; each part
// index carries its job's generation, so a thread still finishing one job
// can never take a part of the next.
class CopyPool {
public:
    static CopyPool& get()
    {
        static CopyPool pool;
        return pool;
    }
    void copy(void* dst, const void* src, size_t bytes)
    {
        std::lock_guard<std::mutex> one_job(job_mu_);
        if (workers_.empty() || bytes < (size_t(1) << 20)) {
            std::memcpy(dst, src, bytes);
            return;
        }
        const int parts = 4 * ((int)workers_.size() + 1);
        {
            std::lock_guard<std::mutex> lk(mu_);
            job_ = Job{(char*)dst, (const char*)src, bytes, parts};
            ++gen_;
            pending_ = parts;
            next_.store(gen_ << 32);
        }
        cv_.notify_all();
        work(gen_, job_);
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [&] { return pending_ == 0; });
    }
    ~CopyPool()
    {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (std::thread& t : workers_)
            t.join();
    }

private:
    struct Job {
        char* dst;
        const char* src;
        size_t bytes;
        int parts;
    };
    CopyPool()
    {
        const unsigned hc = std::thread::hardware_concurrency();
        // besides the caller: half the host's threads, at most 7
        const int n = std::max(0, std::min(7, (int)hc / 2 - 1));
        for (int i = 0; i < n; ++i)
            workers_.emplace_back([this] { loop(); });
    }
    void work(unsigned long long gen, Job job)
    {
        for (;;) {
            unsigned long long v = next_.load();
            if ((v >> 32) != gen || (long long)(v & 0xffffffffu) >= job.parts)
                return;
            if (!next_.compare_exchange_weak(v, v + 1))
                continue;
            const size_t p = v & 0xffffffffu;
            const size_t a = job.bytes * p / job.parts, b = job.bytes * (p + 1) / job.parts;
            std::memcpy(job.dst + a, job.src + a, b - a);
            std::lock_guard<std::mutex> lk(mu_);
            if (--pending_ == 0)
                done_cv_.notify_all();
        }
    }
    void loop()
    {
        unsigned long long seen = 0;
        for (;;) {
            Job job;
            unsigned long long gen;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
                if (stop_)
                    return;
                seen = gen = gen_;
                job = job_;
            }
            work(gen, job);
        }
    }
    std::vector<std::thread> workers_;
    std::mutex job_mu_, mu_;
    std::condition_variable cv_, done_cv_;
    Job job_{};
    unsigned long long gen_ = 0;
    int pending_ = 0;
    bool stop_ = false;
    std::atomic<unsigned long long> next_{0};
};

constexpr size_t kPinChunk = size_t(8) << 20;  // bytes per staging buffer

int ensure_staging(arc_sim* s)
{
    for (int k = 0; k < 2; ++k) {
        if (!s->pin[k] && check(s, cudaMallocHost(&s->pin[k], kPinChunk), "cudaMallocHost(staging)"))
            return ARC_ERR_CUDA;
        if (!s->pin_ev[k] && check(s, cudaEventCreateWithFlags(&s->pin_ev[k], cudaEventDisableTiming), "event"))
            return ARC_ERR_CUDA;
    }
    return ARC_OK;
}

// Device-to-host copy on the sim's stream of `n_seg` consecutive pieces of
// the device range starting at `src` into the host arrays seg_dst[k] (which
// may be pageable) of seg_bytes[k] bytes each, returning when they hold the
// data. Large copies go through two page-locked buffers: the DMA of one chunk
// overlaps the host copy of the one before, which is split over the copy
// threads. Anything queued on the stream before runs first.
int copy_out_pieces(const arc_sim* sc, const void* src, int n_seg, void* const* seg_dst, const size_t* seg_bytes,
                    const char* where)
{
    arc_sim* s = const_cast<arc_sim*>(sc);
    size_t bytes = 0;
    for (int k = 0; k < n_seg; ++k)
        bytes += seg_bytes[k];
    if (bytes < (size_t(2) << 20)) {
        size_t off = 0;
        for (int k = 0; k < n_seg; ++k) {
            if (seg_bytes[k] && check(s, cudaMemcpyAsync(seg_dst[k], (const char*)src + off, seg_bytes[k],
                                                         cudaMemcpyDeviceToHost, s->stream),
                                      where))
                return ARC_ERR_CUDA;
            off += seg_bytes[k];
        }
        return sync(s, where);
    }
    if (ensure_staging(s))
        return ARC_ERR_CUDA;
    const size_t chunks = (bytes + kPinChunk - 1) / kPinChunk;
    auto issue = [&](size_t c) {
        const size_t off = c * kPinChunk, len = std::min(kPinChunk, bytes - off);
        return check(s, cudaMemcpyAsync(s->pin[c & 1], (const char*)src + off, len, cudaMemcpyDeviceToHost, s->stream),
                     where) ||
               check(s, cudaEventRecord(s->pin_ev[c & 1], s->stream), where);
    };
    if (issue(0))
        return ARC_ERR_CUDA;
    int seg = 0;
    size_t seg_start = 0;  // offset of piece `seg` in the device range
    for (size_t c = 0; c < chunks; ++c) {
        // chunk c + 1 goes into the buffer whose host copy finished last round
        if (c + 1 < chunks && issue(c + 1))
            return ARC_ERR_CUDA;
        if (check(s, cudaEventSynchronize(s->pin_ev[c & 1]), where))
            return ARC_ERR_CUDA;
        const size_t off = c * kPinChunk, end = off + std::min(kPinChunk, bytes - off);
        // scatter [off, end) into the pieces it overlaps
        while (seg < n_seg && seg_start + seg_bytes[seg] <= off) {
            seg_start += seg_bytes[seg];
            ++seg;
        }
        size_t ks = seg_start;  // offset of piece k
        for (int k = seg; k < n_seg && ks < end; ks += seg_bytes[k], ++k) {
            const size_t a = std::max(ks, off), b = std::min(ks + seg_bytes[k], end);
            if (b > a)
                CopyPool::get().copy((char*)seg_dst[k] + (a - ks), (const char*)s->pin[c & 1] + (a - off), b - a);
        }
    }
    return ARC_OK;
}

int copy_out(const arc_sim* s, void* dst, const void* src, size_t bytes, const char* where)
{
    return copy_out_pieces(s, src, 1, &dst, &bytes, where);
}

template <class R> const DevModel<R>& dev_model(const arc_sim* s);
template <> const DevModel<float>& dev_model<float>(const arc_sim* s) { return s->mf; }
template <> const DevModel<double>& dev_model<double>(const arc_sim* s) { return s->md; }

// the warp-per-leg step in the sim's precision (FP64: the whole control
// step in one launch; substep tiles are FP32 only)
template <class R> cudaError_t launch_warps(arc_sim*, const DevModel<R>&, const Worlds<R>&, const Actuation&,
                                           const int*, int, int*, cudaStream_t);
template <> cudaError_t launch_warps<float>(arc_sim* s, const DevModel<float>& M, const Worlds<float>& W,
                                            const Actuation& A, const int* ids, int n_items, int* queue,
                                            cudaStream_t st)
{
    return launch_step_warps(M, W, A, static_cast<float*>(s->spill), s->spill_per_lane, s->lane_cap, ids, n_items,
                             queue, st, s->substep_tile, s->tile_q);
}
template <> cudaError_t launch_warps<double>(arc_sim* s, const DevModel<double>& M, const Worlds<double>& W,
                                             const Actuation& A, const int* ids, int n_items, int* queue,
                                             cudaStream_t st)
{
    return launch_step_warps64(M, W, A, static_cast<double*>(s->spill), s->spill_per_lane, s->lane_cap, ids,
                               n_items, queue, st);
}

// ids: device list of n_ids distinct worlds to step (NULL: all worlds).
// A subset is stepped by the warp-per-leg kernel (FP32 quadruped) or the
// plain kernel; the leg-parallel kernel steps whole batches only. part >= 0:
// the worlds of that part of arc_env_step_part, whose launches may run
// beside other parts' and so take their own work queue.
template <class R> int step_impl(arc_sim* s, const Actuation& A, cudaStream_t st, const int* ids, int n_ids, int part)
{
    int* queue = !s->use_queue ? nullptr : (part >= 0 ? s->part_queue + 2 * part : s->queue);
    const Worlds<R> W = view<R>(s);
    const DevModel<R>& M = dev_model<R>(s);
    const int n_items = ids ? n_ids : s->n;
    const bool warps_ok = M.leaper && s->substeps <= kFastMaxSubsteps;
    cudaError_t e;
    if (warps_ok && (s->kernel == ARC_KERNEL_WARPS || (ids && s->kernel == ARC_KERNEL_LEGS)))
        e = launch_warps<R>(s, M, W, A, ids, n_items, queue, st);
    else if (!ids && s->kernel == ARC_KERNEL_LEGS && M.leaper && s->substeps <= kFastMaxSubsteps)
        e = launch_step_fast<R>(M, W, A, static_cast<R*>(s->spill), s->spill_per_lane, s->lane_cap, s->wpc, st);
    else
        e = launch_step_plain<R>(M, W, A, ids, n_items, st);
    return check(s, e, "step kernel");
}

int step_any(arc_sim* s, const Actuation& A, cudaStream_t st, const int* ids = nullptr, int n_ids = 0, int part = -1)
{
    return s->fp64 ? step_impl<double>(s, A, st, ids, n_ids, part) : step_impl<float>(s, A, st, ids, n_ids, part);
}

cudaStream_t stream_of(const arc_sim* s, void* stream) { return stream ? (cudaStream_t)stream : s->stream; }

}  // namespace

// ============================================================================
// Part 1: the reference API

extern "C" {

arc_sim* arc_sim_create(int n_worlds, double dt, int substeps, int grid, double cell)
{
    return arc_sim_create_ex(n_worlds, dt, substeps, grid, cell, 0u);
}

arc_sim* arc_sim_create_ex(int n_worlds, double dt, int substeps, int grid, double cell, unsigned flags)
{
    ModelHost m;
    build_leaper(m);
    return create_with_model(m, n_worlds, dt, substeps, grid, cell, flags);
}

void arc_sim_destroy(arc_sim* s)
{
    if (!s)
        return;
    if (s->stream)
        cudaStreamSynchronize(s->stream);
    free_all(s);
    delete s;
}

void arc_sim_set_threads(arc_sim* s, int threads) { s->threads = threads > 0 ? threads : 1; }
int arc_sim_num_worlds(const arc_sim* s) { return s->n; }
int arc_sim_num_joints(void) { return kNumJoints; }
int arc_sim_num_legs(void) { return kNumLegs; }

void arc_sim_robot_info(const arc_sim* s, double* default_angles, double* lo, double* hi, double* misc)
{
    const ModelHost& m = s->model;
    for (int i = 0; i < kNumJoints && i < m.nj; ++i) {
        if (default_angles)
            default_angles[i] = m.default_angles[i];
        if (lo)
            lo[i] = m.j[i].lo;
        if (hi)
            hi[i] = m.j[i].hi;
    }
    if (misc) {
        misc[0] = m.stand_height;
        misc[1] = m.total_mass;
    }
}

void arc_sim_reset(arc_sim* s, const int* ids, int n_ids, const unsigned int* seeds, const double* difficulty)
{
    if (n_ids <= 0)
        return;
    if (!ids_ok(s, ids, n_ids)) {
        fail(s, ARC_ERR_ARG, "arc_sim_reset: world index out of range");
        return;
    }
    // one staging block: difficulty (8-byte aligned) first, then ids and seeds
    char* buf = (char*)grow(s, s->st_in, (size_t)n_ids * (sizeof(double) + sizeof(int) + sizeof(unsigned)));
    if (!buf)
        return;
    double* d_diff = (double*)buf;
    int* d_ids = (int*)(buf + (size_t)n_ids * sizeof(double));
    unsigned* d_seeds = (unsigned*)(buf + (size_t)n_ids * (sizeof(double) + sizeof(int)));
    cudaStream_t st = s->stream;
    if (check(s, cudaMemcpyAsync(d_ids, ids, sizeof(int) * n_ids, cudaMemcpyHostToDevice, st), "reset ids") ||
        check(s, cudaMemcpyAsync(d_seeds, seeds, sizeof(unsigned) * n_ids, cudaMemcpyHostToDevice, st), "seeds") ||
        check(s, cudaMemcpyAsync(d_diff, difficulty, sizeof(double) * n_ids, cudaMemcpyHostToDevice, st), "diff"))
        return;
    cudaError_t e;
    if (s->fp64)
        e = launch_reset_warp<double>(s->rm, view<double>(s), (TerrainGeom<double>*)s->tg, s->tgd, d_ids, n_ids,
                                      d_seeds, d_diff, s->grid_of, s->cell, st);
    else
        e = launch_reset_warp<float>(s->rm, view<float>(s), (TerrainGeom<float>*)s->tg, s->tgd, d_ids, n_ids,
                                     d_seeds, d_diff, s->grid_of, s->cell, st);
    if (check(s, e, "reset kernel"))
        return;
    sync(s, "arc_sim_reset");
}

void arc_sim_step(arc_sim* s, const double* targets)
{
    if (s->n <= 0)
        return;
    const size_t bytes = sizeof(double) * (size_t)s->n * kNumJoints;
    double* d = (double*)grow(s, s->st_in2, bytes);
    if (!d)
        return;
    if (check(s, cudaMemcpyAsync(d, targets, bytes, cudaMemcpyHostToDevice, s->stream), "step targets"))
        return;
    Actuation A{d, nullptr};
    if (step_any(s, A, s->stream))
        return;
    sync(s, "arc_sim_step");
}

void arc_sim_observe(const arc_sim* s, double* root, double* rot, double* joints, double* contacts, int* flags)
{
    if (s->n <= 0)
        return;
    const size_t n = (size_t)s->n;
    const int nch = s->model.n_channels;
    const size_t sizes[5] = {n * 13, n * 9, n * 3 * s->model.nj, n * nch, n};
    double* outs[4] = {root, rot, joints, contacts};
    size_t total = sizes[0] + sizes[1] + sizes[2] + sizes[3] + sizes[4];
    double* d = (double*)grow(s, const_cast<arc_sim*>(s)->st_out, total * sizeof(double));
    if (!d)
        return;
    double* dr = d;
    double* drot = dr + sizes[0];
    double* dj = drot + sizes[1];
    double* dc = dj + sizes[2];
    int* df = (int*)(dc + sizes[3]);
    cudaError_t e;
    if (s->fp64)
        e = launch_observe<double>(s->md, view<double>(s), root ? dr : nullptr, rot ? drot : nullptr,
                                   joints ? dj : nullptr, contacts ? dc : nullptr, flags ? df : nullptr, s->stream);
    else
        e = launch_observe<float>(s->mf, view<float>(s), root ? dr : nullptr, rot ? drot : nullptr,
                                  joints ? dj : nullptr, contacts ? dc : nullptr, flags ? df : nullptr, s->stream);
    if (check(s, e, "observe kernel"))
        return;
    // the five outputs lie back to back on the device: one staged copy; a
    // NULL output's bytes go to a scratch array
    std::vector<char>& skip = const_cast<arc_sim*>(s)->skip;
    size_t skip_bytes = 0;
    for (int k = 0; k < 5; ++k)
        if (!(k < 4 ? (void*)outs[k] : (void*)flags))
            skip_bytes = std::max(skip_bytes, sizes[k] * (k < 4 ? sizeof(double) : sizeof(int)));
    if (skip.size() < skip_bytes)
        skip.resize(skip_bytes);
    void* dsts[5];
    size_t lens[5];
    for (int k = 0; k < 5; ++k) {
        void* o = k < 4 ? (void*)outs[k] : (void*)flags;
        dsts[k] = o ? o : (void*)skip.data();
        lens[k] = sizes[k] * (k < 4 ? sizeof(double) : sizeof(int));
    }
    copy_out_pieces(s, d, 5, dsts, lens, "arc_sim_observe");
}

void arc_sim_heights(const arc_sim* s, const double* offsets, int k, double* out)
{
    if (s->n <= 0 || k <= 0)
        return;
    arc_sim* m = const_cast<arc_sim*>(s);
    double* doff = (double*)grow(s, m->st_in3, sizeof(double) * 2 * k);
    double* dout = (double*)grow(s, m->st_out, sizeof(double) * (size_t)s->n * k);
    if (!doff || !dout)
        return;
    if (check(s, cudaMemcpyAsync(doff, offsets, sizeof(double) * 2 * k, cudaMemcpyHostToDevice, s->stream), "offs"))
        return;
    cudaError_t e = s->fp64 ? launch_heights<double>(view<double>(s), doff, k, dout, s->stream)
                            : launch_heights<float>(view<float>(s), doff, k, dout, s->stream);
    if (check(s, e, "heights kernel"))
        return;
    copy_out(s, out, dout, sizeof(double) * (size_t)s->n * k, "heights copy");
}

void arc_sim_terrain_at(const arc_sim* s, const int* ids, const double* xy, int m, double* out)
{
    if (m <= 0)
        return;
    if (!ids_ok(s, ids, m)) {
        fail(s, ARC_ERR_ARG, "arc_sim_terrain_at: world index out of range");
        return;
    }
    arc_sim* ms = const_cast<arc_sim*>(s);
    char* buf = (char*)grow(s, ms->st_in3, (size_t)m * (sizeof(int) + 3 * sizeof(double)) + 64);
    if (!buf)
        return;
    double* dxy = (double*)buf;
    double* dout = dxy + 2 * (size_t)m;
    int* dids = (int*)(dout + m);
    if (check(s, cudaMemcpyAsync(dids, ids, sizeof(int) * m, cudaMemcpyHostToDevice, s->stream), "ids") ||
        check(s, cudaMemcpyAsync(dxy, xy, sizeof(double) * 2 * m, cudaMemcpyHostToDevice, s->stream), "xy"))
        return;
    cudaError_t e = s->fp64 ? launch_terrain_at<double>(view<double>(s), dids, dxy, m, dout, s->stream)
                            : launch_terrain_at<float>(view<float>(s), dids, dxy, m, dout, s->stream);
    if (check(s, e, "terrain_at kernel"))
        return;
    if (check(s, cudaMemcpyAsync(out, dout, sizeof(double) * m, cudaMemcpyDeviceToHost, s->stream), "out"))
        return;
    sync(s, "arc_sim_terrain_at");
}

const arc_world* arc_sim_world(const arc_sim* s, int i)
{
    if (i < 0 || i >= s->n) {
        fail(s, ARC_ERR_ARG, "arc_sim_world: world index out of range");
        return nullptr;
    }
    arc_sim* ms = const_cast<arc_sim*>(s);
    if (!ms->hworld)
        ms->hworld = new arc_world();
    arc_world* w = ms->hworld;
    std::memset(w, 0, sizeof(*w));
    const ModelHost& m = s->model;
    std::vector<double> st(arc_sim_state_size(s));
    if (arc_sim_get_state(s, &i, 1, st.data()) != ARC_OK)
        return nullptr;
    int nxy[2];
    double geom[4];
    std::vector<double> h(kGridMax * kGridMax);
    if (arc_sim_get_terrain(s, i, nxy, geom, h.data()) != ARC_OK)
        return nullptr;
    w->gravity = arcw_vec3{m.gravity.x, m.gravity.y, m.gravity.z};
    w->mu_static = m.mu_s;
    w->mu_dynamic = m.mu_d;
    w->n_bodies = m.nb;
    w->n_joints = m.nj;
    w->n_spheres = m.ns;
    const double* p = st.data();
    for (int b = 0; b < m.nb; ++b, p += 13) {
        arcw_body& o = w->bodies[b];
        o.x = o.x_prev = arcw_vec3{p[0], p[1], p[2]};
        o.q = o.q_prev = arcw_quat{p[3], p[4], p[5], p[6]};
        o.v = arcw_vec3{p[7], p[8], p[9]};
        o.w = arcw_vec3{p[10], p[11], p[12]};
        o.mass = m.b[b].mass;
        o.inv_mass = m.b[b].inv_mass;
        o.inertia = arcw_vec3{m.b[b].inertia.x, m.b[b].inertia.y, m.b[b].inertia.z};
        o.inv_inertia = arcw_vec3{m.b[b].inv_inertia.x, m.b[b].inv_inertia.y, m.b[b].inv_inertia.z};
        Pose<double> P;
        P.q = Q4<double>{p[3], p[4], p[5], p[6]};
        BodyK<double> k{m.b[b].inv_mass, m.b[b].inertia, m.b[b].inv_inertia,
                        m.b[b].inertia.x == m.b[b].inertia.y && m.b[b].inertia.y == m.b[b].inertia.z};
        body_sync(P, k);
        for (int a = 0; a < 3; ++a)
            for (int c = 0; c < 3; ++c)
                o.rot.m[a][c] = P.rot.m[a][c];
        double iw[3][3] = {{P.iiw.xx, P.iiw.xy, P.iiw.xz}, {P.iiw.xy, P.iiw.yy, P.iiw.yz},
                           {P.iiw.xz, P.iiw.yz, P.iiw.zz}};
        std::memcpy(o.inv_iw.m, iw, sizeof(iw));
    }
    for (int sidx = 0; sidx < m.ns; ++sidx, p += 8) {
        arcw_sphere& o = w->spheres[sidx];
        o.body = m.s[sidx].body;
        o.pos = arcw_vec3{m.s[sidx].pos.x, m.s[sidx].pos.y, m.s[sidx].pos.z};
        o.radius = m.s[sidx].radius;
        o.anchored = p[0] != 0.0;
        o.anchor = arcw_vec3{p[1], p[2], p[3]};
        o.anchor_n = arcw_vec3{p[4], p[5], p[6]};
        o.touch = (int)p[7];
    }
    for (int j = 0; j < m.nj; ++j, p += 4) {
        arcw_joint& o = w->joints[j];
        const ModelHost::Joint& t = m.j[j];
        o.parent = t.parent;
        o.child = t.child;
        o.r1 = arcw_vec3{t.r1.x, t.r1.y, t.r1.z};
        o.r2 = arcw_vec3{t.r2.x, t.r2.y, t.r2.z};
        o.a1 = arcw_vec3{t.a1.x, t.a1.y, t.a1.z};
        o.a2 = arcw_vec3{t.a2.x, t.a2.y, t.a2.z};
        o.b1 = arcw_vec3{t.b1.x, t.b1.y, t.b1.z};
        o.b2 = arcw_vec3{t.b2.x, t.b2.y, t.b2.z};
        o.q_rel0 = arcw_quat{t.q_rel0.w, t.q_rel0.x, t.q_rel0.y, t.q_rel0.z};
        o.lo = t.lo;
        o.hi = t.hi;
        o.kp = t.kp;
        o.kd = t.kd;
        o.max_torque = t.max_torque;
        o.target = p[0];
        o.angle = p[1];
        o.rate = p[2];
        o.torque = p[3];
        o.lim[0] = std::cos(t.lo);
        o.lim[1] = std::sin(t.lo);
        o.lim[2] = std::cos(t.hi);
        o.lim[3] = std::sin(t.hi);
    }
    // the contact list of the last substep (csrc/arc_phys.c:493-499), once
    // the kernels record it: the first call turns recording on
    if (!s->lastc) {
        arc_sim_set_record_contacts(ms, 1);
    } else {
        const size_t rec = (size_t)kMaxContacts * kContactRec;
        int count = 0;
        std::vector<double> c(rec);
        cudaStream_t st = s->stream;
        bool good = check(s, cudaMemcpyAsync(&count, s->lastn + i, sizeof(int), cudaMemcpyDeviceToHost, st),
                          "contact count") == ARC_OK;
        if (s->fp64) {
            good = good && check(s, cudaMemcpyAsync(c.data(), static_cast<double*>(s->lastc) + (size_t)i * rec,
                                                    sizeof(double) * rec, cudaMemcpyDeviceToHost, st),
                                 "contacts") == ARC_OK;
            good = good && check(s, cudaStreamSynchronize(st), "contacts") == ARC_OK;
        } else {
            std::vector<float> f(rec);
            good = good && check(s, cudaMemcpyAsync(f.data(), static_cast<float*>(s->lastc) + (size_t)i * rec,
                                                    sizeof(float) * rec, cudaMemcpyDeviceToHost, st),
                                 "contacts") == ARC_OK;
            good = good && check(s, cudaStreamSynchronize(st), "contacts") == ARC_OK;
            for (size_t k = 0; k < rec; ++k)
                c[k] = f[k];
        }
        if (!good)
            return nullptr;
        w->n_contacts = std::max(0, std::min(count, kMaxContacts));
        for (int k = 0; k < w->n_contacts; ++k) {
            const double* r = c.data() + (size_t)k * kContactRec;
            w->contacts[k].body = (int)r[0];
            w->contacts[k].local = arcw_vec3{r[1], r[2], r[3]};
            w->contacts[k].n = arcw_vec3{r[4], r[5], r[6]};
        }
    }
    w->n_visuals = m.nv;
    for (int k = 0; k < m.nv; ++k) {
        const ModelHost::Visual& v = m.v[k];
        arcw_visual& o = w->visuals[k];
        o.type = v.type;
        o.body = v.body;
        o.p0 = arcw_vec3{v.p0.x, v.p0.y, v.p0.z};
        o.p1 = arcw_vec3{v.p1.x, v.p1.y, v.p1.z};
        o.radius = v.radius;
        o.radius2 = v.radius2;
        o.aspect = v.aspect;
        o.material = v.material;
        std::memcpy(o.color, v.color, sizeof(o.color));
    }
    w->unstable = p[0] != 0.0;
    w->time = p[1];
    w->terrain.nx = nxy[0];
    w->terrain.ny = nxy[1];
    w->terrain.cell = geom[0];
    w->terrain.ox = geom[1];
    w->terrain.oy = geom[2];
    w->terrain.outside = geom[3];
    std::memcpy(w->terrain.h, h.data(), sizeof(double) * nxy[0] * nxy[1]);
    return w;
}

// ============================================================================
// Part 2: additive API

int arc_sim_last_error(const arc_sim* s) { return s ? s->err : ARC_ERR_ARG; }
const char* arc_sim_error_message(const arc_sim* s) { return s ? s->msg.c_str() : "null sim"; }

int arc_sim_set_kernel(arc_sim* s, int kernel, int worlds_per_cta)
{
    if (kernel == ARC_KERNEL_LEGS) {
        if (!s->model.leaper)
            return fail(s, ARC_ERR_UNSUPPORTED, "leg-parallel kernel needs the quadruped's topology");
        if (worlds_per_cta != 1 && worlds_per_cta != 2 && worlds_per_cta != 4 && worlds_per_cta != 8 &&
            worlds_per_cta != 16 && worlds_per_cta != 32 && worlds_per_cta != 64)
            return fail(s, ARC_ERR_ARG, "worlds_per_cta must be 1, 2, 4, 8, 16, 32 or 64");
        const size_t smem = s->fp64 ? fast_smem_bytes<double>(s->stride, worlds_per_cta)
                                    : fast_smem_bytes<float>(s->stride, worlds_per_cta);
        if (smem > 227 * 1024)
            return fail(s, ARC_ERR_UNSUPPORTED, "worlds_per_cta needs more than 227 KB of shared memory");
        s->wpc = worlds_per_cta;
    } else if (kernel == ARC_KERNEL_WARPS) {
        if (!s->model.leaper)
            return fail(s, ARC_ERR_UNSUPPORTED, "warp-per-leg kernel needs the quadruped's topology");
    } else if (kernel != ARC_KERNEL_PLAIN) {
        return fail(s, ARC_ERR_ARG, "unknown kernel");
    }
    s->kernel = kernel;
    return ARC_OK;
}

int arc_sim_get_kernel(const arc_sim* s, int* kernel, int* worlds_per_cta)
{
    if (kernel)
        *kernel = s->kernel;
    if (worlds_per_cta)
        *worlds_per_cta = s->kernel == ARC_KERNEL_WARPS ? 32 : (s->kernel == ARC_KERNEL_PLAIN ? 1 : s->wpc);
    return ARC_OK;
}

int arc_sim_real_size(const arc_sim* s) { return real_size(s); }

int arc_sim_model_info(const arc_sim* s, int* n_bodies, int* n_joints, int* n_spheres, int* n_channels)
{
    if (n_bodies)
        *n_bodies = s->model.nb;
    if (n_joints)
        *n_joints = s->model.nj;
    if (n_spheres)
        *n_spheres = s->model.ns;
    if (n_channels)
        *n_channels = s->model.n_channels;
    return ARC_OK;
}

int arc_sim_state_size(const arc_sim* s)
{
    return s->model.nb * 13 + s->model.ns * 8 + s->model.nj * 4 + 2;
}

int arc_sim_get_state(const arc_sim* s, const int* ids, int n_ids, double* out)
{
    if (n_ids <= 0)
        return ARC_OK;
    if (!ids_ok(s, ids, n_ids))
        return fail(s, ARC_ERR_ARG, "arc_sim_get_state: world index out of range");
    arc_sim* m = const_cast<arc_sim*>(s);
    const size_t ss = arc_sim_state_size(s);
    int* dids = (int*)grow(s, m->st_in3, sizeof(int) * n_ids);
    double* dout = (double*)grow(s, m->st_out, sizeof(double) * ss * n_ids);
    if (!dids || !dout)
        return ARC_ERR_CUDA;
    if (check(s, cudaMemcpyAsync(dids, ids, sizeof(int) * n_ids, cudaMemcpyHostToDevice, s->stream), "ids"))
        return ARC_ERR_CUDA;
    cudaError_t e = s->fp64 ? launch_get_state<double>(s->md, view<double>(s), dids, n_ids, dout, s->stream)
                            : launch_get_state<float>(s->mf, view<float>(s), dids, n_ids, dout, s->stream);
    if (check(s, e, "get_state kernel"))
        return ARC_ERR_CUDA;
    return copy_out(s, out, dout, sizeof(double) * ss * n_ids, "arc_sim_get_state");
}

int arc_sim_set_state(arc_sim* s, const int* ids, int n_ids, const double* in)
{
    if (n_ids <= 0)
        return ARC_OK;
    if (!ids_ok(s, ids, n_ids))
        return fail(s, ARC_ERR_ARG, "arc_sim_set_state: world index out of range");
    const size_t ss = arc_sim_state_size(s);
    int* dids = (int*)grow(s, s->st_in3, sizeof(int) * n_ids);
    double* din = (double*)grow(s, s->st_in, sizeof(double) * ss * n_ids);
    if (!dids || !din)
        return ARC_ERR_CUDA;
    if (check(s, cudaMemcpyAsync(dids, ids, sizeof(int) * n_ids, cudaMemcpyHostToDevice, s->stream), "ids") ||
        check(s, cudaMemcpyAsync(din, in, sizeof(double) * ss * n_ids, cudaMemcpyHostToDevice, s->stream), "in"))
        return ARC_ERR_CUDA;
    cudaError_t e = s->fp64 ? launch_set_state<double>(s->md, view<double>(s), dids, n_ids, din, s->stream)
                            : launch_set_state<float>(s->mf, view<float>(s), dids, n_ids, din, s->stream);
    if (check(s, e, "set_state kernel"))
        return ARC_ERR_CUDA;
    return sync(s, "arc_sim_set_state");
}

int arc_sim_set_terrain(arc_sim* s, int id, int nx, int ny, double cell, double outside, const double* heights)
{
    if (id < 0 || id >= s->n || nx <= 0 || ny <= 0 || nx > kGridMax || ny > kGridMax || !(cell > 0.0))
        return fail(s, ARC_ERR_ARG, "arc_sim_set_terrain: bad world index or grid size");
    if ((long long)nx * ny > (long long)s->grid_host[id] * s->grid_host[id])
        return fail(s, ARC_ERR_ARG, "arc_sim_set_terrain: more columns than the world's terrain holds");
    if (ensure_spill(s, cell) != ARC_OK)
        return ARC_ERR_CUDA;
    double* d = (double*)grow(s, s->st_in, sizeof(double) * nx * ny);
    if (!d)
        return ARC_ERR_CUDA;
    if (check(s, cudaMemcpyAsync(d, heights, sizeof(double) * nx * ny, cudaMemcpyHostToDevice, s->stream), "h"))
        return ARC_ERR_CUDA;
    cudaError_t e = s->fp64 ? launch_set_terrain<double>(view<double>(s), (TerrainGeom<double>*)s->tg, s->tgd, id,
                                                         nx, ny, cell, outside, d, s->stream)
                            : launch_set_terrain<float>(view<float>(s), (TerrainGeom<float>*)s->tg, s->tgd, id, nx,
                                                        ny, cell, outside, d, s->stream);
    if (check(s, e, "set_terrain kernel"))
        return ARC_ERR_CUDA;
    return sync(s, "arc_sim_set_terrain");
}

int arc_sim_get_terrain(const arc_sim* s, int id, int* nx_ny, double* geom, double* heights)
{
    if (id < 0 || id >= s->n)
        return fail(s, ARC_ERR_ARG, "arc_sim_get_terrain: world index out of range");
    TerrainGeomD g;
    long long off = 0;
    if (check(s, cudaMemcpyAsync(&g, s->tgd + id, sizeof(g), cudaMemcpyDeviceToHost, s->stream), "geom") ||
        check(s, cudaMemcpyAsync(&off, s->toff + id, sizeof(off), cudaMemcpyDeviceToHost, s->stream), "off") ||
        sync(s, "get_terrain"))
        return ARC_ERR_CUDA;
    if (nx_ny) {
        nx_ny[0] = g.nx;
        nx_ny[1] = g.ny;
    }
    if (geom) {
        geom[0] = g.cell;
        geom[1] = g.ox;
        geom[2] = g.oy;
        geom[3] = g.outside;
    }
    if (heights) {
        const int cnt = g.nx * g.ny;
        if (s->fp64) {
            if (check(s, cudaMemcpy(heights, (double*)s->th + off, sizeof(double) * cnt, cudaMemcpyDeviceToHost),
                      "heights"))
                return ARC_ERR_CUDA;
        } else {
            std::vector<float> tmp(cnt);
            if (check(s, cudaMemcpy(tmp.data(), (float*)s->th + off, sizeof(float) * cnt, cudaMemcpyDeviceToHost),
                      "heights"))
                return ARC_ERR_CUDA;
            for (int c = 0; c < cnt; ++c)
                heights[c] = tmp[c];
        }
    }
    return ARC_OK;
}

int arc_sim_set_world_params(arc_sim* s, const double* gravity, double mu_static, double mu_dynamic)
{
    if (gravity)
        s->model.gravity = V3<double>{gravity[0], gravity[1], gravity[2]};
    s->model.mu_s = mu_static;
    s->model.mu_d = mu_dynamic;
    rebuild_models(s);
    return ARC_OK;
}

int arc_sim_set_joint(arc_sim* s, int j, double lo, double hi, double kp, double kd, double max_torque)
{
    if (j < 0 || j >= s->model.nj)
        return fail(s, ARC_ERR_ARG, "arc_sim_set_joint: joint index out of range");
    ModelHost::Joint& t = s->model.j[j];
    t.lo = lo;
    t.hi = hi;
    t.kp = kp;
    t.kd = kd;
    t.max_torque = max_torque;
    rebuild_models(s);
    return ARC_OK;
}

arc_model* arc_model_create(void)
{
    arc_model* m = new arc_model();
    m->m.n_channels = 1;
    return m;
}

void arc_model_destroy(arc_model* m) { delete m; }

int arc_model_add_body(arc_model* m, double mass, const double* inertia, const double* pos, const double* q)
{
    return m->m.add_body(mass, V3<double>{inertia[0], inertia[1], inertia[2]}, V3<double>{pos[0], pos[1], pos[2]},
                         Q4<double>{q[0], q[1], q[2], q[3]});
}

int arc_model_add_sphere(arc_model* m, int body, const double* local_pos, double radius)
{
    if (body < 0 || body >= m->m.nb)
        return -1;
    return m->m.add_sphere(body, V3<double>{local_pos[0], local_pos[1], local_pos[2]}, radius);
}

int arc_model_add_hinge(arc_model* m, int parent, int child, const double* anchor, const double* axis)
{
    if (child < 0 || child >= m->m.nb || parent >= m->m.nb)
        return -1;
    return m->m.add_hinge(parent, child, V3<double>{anchor[0], anchor[1], anchor[2]},
                          V3<double>{axis[0], axis[1], axis[2]});
}

int arc_model_add_visual(arc_model* m, int type, int body, const double* p0, const double* p1, double radius,
                         double radius2, double aspect, int material, const float* rgb)
{
    if (!m || body < 0 || body >= m->m.nb || type < kVisSphere || type > kVisRing || material < kMatPaint ||
        material > kMatGlow || !p0 || !p1 || !rgb)
        return -1;
    int i = m->m.add_visual(type, body, V3<double>{p0[0], p0[1], p0[2]}, V3<double>{p1[0], p1[1], p1[2]}, radius,
                            radius2, material, rgb);
    if (i >= 0)
        m->m.v[i].aspect = aspect;
    return i;
}

arc_sim* arc_sim_create_model(const arc_model* m, int n_worlds, double dt, int substeps, int grid, double cell,
                              unsigned flags)
{
    if (!m || m->m.nb <= 0)
        return nullptr;
    ModelHost model = m->m;
    for (int j = 0; j < model.nj; ++j)
        model.default_angles[j] = 0.0;
    return create_with_model(model, n_worlds, dt, substeps, grid, cell, flags | ARC_SIM_PLAIN);
}

int arc_sim_set_pose(arc_sim* s, int id, const double* pos, const double* q, const double* angles)
{
    if (id < 0 || id >= s->n)
        return fail(s, ARC_ERR_ARG, "arc_sim_set_pose: world index out of range");
    const ModelHost& m = s->model;
    std::vector<double> st(arc_sim_state_size(s));
    int rc = arc_sim_get_state(s, &id, 1, st.data());
    if (rc != ARC_OK)
        return rc;
    V3<double> xs[kMaxBodies];
    Q4<double> qs[kMaxBodies];
    std::vector<double> zero(kMaxJoints, 0.0);
    const double* ang = angles ? angles : zero.data();
    m.pose(V3<double>{pos[0], pos[1], pos[2]}, Q4<double>{q[0], q[1], q[2], q[3]}, ang, xs, qs);
    double* p = st.data();
    for (int b = 0; b < m.nb; ++b, p += 13) {
        p[0] = xs[b].x; p[1] = xs[b].y; p[2] = xs[b].z;
        p[3] = qs[b].w; p[4] = qs[b].x; p[5] = qs[b].y; p[6] = qs[b].z;
        for (int c = 7; c < 13; ++c)
            p[c] = 0.0;
    }
    for (int sidx = 0; sidx < m.ns; ++sidx, p += 8) {
        p[0] = 0.0;  // anchored
        p[7] = 0.0;  // touch
    }
    for (int j = 0; j < m.nj; ++j, p += 4) {
        p[0] = ang[j];
        p[1] = ang[j];
        p[2] = 0.0;
        p[3] = 0.0;
    }
    p[0] = 0.0;  // unstable; time is kept
    return arc_sim_set_state(s, &id, 1, st.data());
}

void* arc_sim_stream(const arc_sim* s) { return (void*)s->stream; }

int arc_sim_step_device(arc_sim* s, const double* d_targets, void* stream)
{
    Actuation A{d_targets, nullptr};
    return step_any(s, A, stream_of(s, stream));
}

int arc_sim_step_actions(arc_sim* s, const float* d_actions, void* stream)
{
    Actuation A{nullptr, d_actions};
    return step_any(s, A, stream_of(s, stream));
}

int arc_sim_step_ids(arc_sim* s, const int* d_ids, int n_ids, const double* d_targets, const float* d_actions,
                     void* stream)
{
    if (n_ids < 0 || (n_ids > 0 && !d_ids) || (!d_targets) == (!d_actions))
        return fail(s, ARC_ERR_ARG, "arc_sim_step_ids: need ids and exactly one of targets, actions");
    if (n_ids == 0)
        return ARC_OK;
    Actuation A{d_targets, d_actions};
    return step_any(s, A, stream_of(s, stream), d_ids, n_ids);
}

int arc_sim_set_work_queue(arc_sim* s, int on)
{
    s->use_queue = on != 0;
    return ARC_OK;
}

int arc_sim_set_record_contacts(arc_sim* s, int on)
{
    if (!on) {
        cudaFree(s->lastc);
        cudaFree(s->lastn);
        s->lastc = nullptr;
        s->lastn = nullptr;
        return ARC_OK;
    }
    if (s->lastc)
        return ARC_OK;
    const size_t n = (size_t)std::max(s->n, 1);
    void* c = nullptr;
    int* k = nullptr;
    if (check(s, cudaMalloc(&c, n * kMaxContacts * kContactRec * real_size(s)), "cudaMalloc(contact lists)"))
        return ARC_ERR_CUDA;
    if (check(s, cudaMalloc((void**)&k, n * sizeof(int)), "cudaMalloc(contact counts)") ||
        check(s, cudaMemsetAsync(k, 0, n * sizeof(int), s->stream), "zero contact counts") ||
        check(s, cudaStreamSynchronize(s->stream), "contact lists")) {
        cudaFree(c);
        cudaFree(k);
        return ARC_ERR_CUDA;
    }
    s->lastc = c;
    s->lastn = k;
    return ARC_OK;
}

int arc_sim_set_substep_tile(arc_sim* s, int tile)
{
    if (tile < 0)
        return fail(s, ARC_ERR_ARG, "arc_sim_set_substep_tile: tile < 0");
    if (s->fp64 && tile > 0 && tile < s->substeps)
        return fail(s, ARC_ERR_UNSUPPORTED, "arc_sim_set_substep_tile: substep tiles are FP32 only");
    if (tile > 0 && tile < s->substeps && !s->tile_q &&
        check(s, cudaMalloc((void**)&s->tile_q, sizeof(float) * 13 * 4 * (size_t)std::max(s->n, 1)),
              "cudaMalloc(tile quaternions)"))
        return ARC_ERR_CUDA;
    s->substep_tile = tile;
    return ARC_OK;
}

int arc_env_set_fused(arc_sim* s, int mode)
{
    if (mode < 0 || mode > 2)
        return fail(s, ARC_ERR_ARG, "arc_env_set_fused: mode 0, 1 or 2");
    s->fused = mode;
    return ARC_OK;
}

int arc_env_set_step_order(arc_sim* s, int mode)
{
    if (mode < 0 || mode > 1)
        return fail(s, ARC_ERR_ARG, "arc_env_set_step_order: mode 0 or 1");
    s->step_order = mode;
    return ARC_OK;
}

int arc_device_checks(unsigned long long* failures, int* first_site, long long* first_index, int clear)
{
    unsigned long long total = 0;
    int site = 0;
    long long index = 0;
#ifdef ARC_DEVICE_CHECKS
    for (auto read : arc::device_check_readers()) {
        unsigned long long r[3];
        if (read(r, clear != 0))
            return ARC_ERR_CUDA;
        total += r[0];
        if (r[0] && !site) {
            site = (int)r[1];
            index = (long long)r[2];
        }
    }
#else
    (void)clear;
#endif
    if (failures)
        *failures = total;
    if (first_site)
        *first_site = site;
    if (first_index)
        *first_index = index;
#ifdef ARC_DEVICE_CHECKS
    return 1;
#else
    return 0;
#endif
}

arc_sim* arc_sim_create_sized(int n_worlds, const int* grids, double dt, int substeps, double cell, unsigned flags)
{
    if (n_worlds < 0 || (n_worlds > 0 && !grids))
        return nullptr;
    int gmax = 1;
    for (int i = 0; i < n_worlds; ++i) {
        if (grids[i] < 1 || grids[i] > kGridMax) {
            std::fprintf(stderr, "arc_sim_create_sized: world %d: grid %d outside 1..%d\n", i, grids[i], kGridMax);
            return nullptr;
        }
        gmax = std::max(gmax, grids[i]);
    }
    ModelHost m;
    build_leaper(m);
    return create_with_model(m, n_worlds, dt, substeps, gmax, cell, flags, grids);
}

int arc_sim_observe_device(const arc_sim* s, double* root, double* rot, double* joints, double* contacts, int* flags,
                           void* stream)
{
    cudaStream_t st = stream_of(s, stream);
    cudaError_t e = s->fp64 ? launch_observe<double>(s->md, view<double>(s), root, rot, joints, contacts, flags, st)
                            : launch_observe<float>(s->mf, view<float>(s), root, rot, joints, contacts, flags, st);
    return check(s, e, "observe kernel");
}

int arc_sim_synchronize(const arc_sim* s) { return sync(s, "arc_sim_synchronize"); }

int arc_sim_observe_ids(const arc_sim* s, const int* d_ids, int n_ids, double* root, double* rot, double* joints,
                        double* contacts, int* flags, void* stream)
{
    if (n_ids < 0 || (n_ids > 0 && !d_ids))
        return fail(s, ARC_ERR_ARG, "arc_sim_observe_ids: need device ids");
    if (n_ids == 0)
        return ARC_OK;
    cudaStream_t st = stream_of(s, stream);
    cudaError_t e = s->fp64 ? launch_observe<double>(s->md, view<double>(s), root, rot, joints, contacts, flags, st,
                                                     d_ids, n_ids)
                            : launch_observe<float>(s->mf, view<float>(s), root, rot, joints, contacts, flags, st,
                                                    d_ids, n_ids);
    return check(s, e, "observe kernel");
}


// ============================================================================
// the task layer on the device

void arc_task_config_default(arc_task_config* c)
{
    // arc/task.py:17-66
    c->dt = 1.0 / 30.0;
    c->max_steps = 1000;
    c->action_scale = 0.6;
    c->checkpoint_radius = 0.5;
    c->checkpoint_min_dist = 3.0;
    c->checkpoint_max_dist = 6.0;
    c->border = 1.5;
    c->w_progress = 10.0;
    c->max_speed = 1.2;
    c->fov = 45.0;
    c->w_turn = 1.0;
    c->w_checkpoint = 10.0;
    c->w_time = 0.05;
    c->w_fall = 20.0;
    c->w_energy = 0.002;
    c->w_action_rate = 0.005;
    c->w_body_contact = 0.02;
    c->w_torso_contact = 0.5;
    c->w_body_rate = 0.01;
    c->w_bounce = 0.05;
    c->flip_up_z = 0.3;
    c->beached_steps = 30;
    c->void_z = -2.0;
    c->curriculum = 1;
    c->difficulty = 0.0;
    c->max_difficulty = 1.0;
    c->level_step = 0.1;
    c->level_up_checkpoints = 3;
    c->level_down_steps = 300;
}

}  // extern "C"

namespace {

template <class T> T* env_alloc(arc_sim* s, size_t count, bool& ok)
{
    void* p = nullptr;
    if (!ok || cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
        ok = false;
        return nullptr;
    }
    cudaMemset(p, 0, std::max<size_t>(count, 1) * sizeof(T));
    s->env_allocs.push_back(p);
    return static_cast<T*>(p);
}

int env_check(const arc_sim* s)
{
    if (!s->env)
        return fail(s, ARC_ERR_ARG, "arc_env_* needs arc_env_init first");
    if (!s->model.leaper)
        return fail(s, ARC_ERR_UNSUPPORTED, "the task layer needs the quadruped model");
    return ARC_OK;
}

template <class R> int env_task_step(arc_sim* s, const float* actions, bool write_obs, cudaStream_t st)
{
    const Worlds<R> W = view<R>(s);
    if (check(s, cudaMemsetAsync(s->to.done_count, 0, sizeof(int), st), "memset done_count"))
        return ARC_ERR_CUDA;
    if (check(s, launch_task_step<R>(dev_model<R>(s), W, s->tp, s->ts, s->to, actions, write_obs ? 2 : 0, st),
              "task step kernel"))
        return ARC_ERR_CUDA;
    return write_obs ? check(s, launch_task_heights<R>(dev_model<R>(s), W, s->tp, s->to, st), "task heights kernel")
                     : ARC_OK;
}

template <class R> int env_reset_done(arc_sim* s, cudaStream_t st)
{
    return check(s,
                 launch_task_reset<R>(dev_model<R>(s), s->rm, view<R>(s), (TerrainGeom<R>*)s->tg, s->tgd, s->grid_of,
                                      s->cell, s->tp, s->ts, s->to.obs, s->to.done_list, s->to.done_count, s->n, st),
                 "task reset kernel");
}

// Whether the env's control step runs fused (the warp-per-leg step and the
// task layer in k_control_step): FP32, the quadruped, that kernel, whole
// control steps.
bool fused_applies(const arc_sim* s)
{
    return s->fused > 0 && !s->fp64 && s->mf.leaper && s->substeps <= kFastMaxSubsteps && s->kernel == ARC_KERNEL_WARPS &&
           (s->substep_tile <= 0 || s->substep_tile >= s->substeps);
}

// The fused control step over ids[0 .. n) (NULL: every world), its ended
// worlds into O's list (O.done_count zeroed first) and reset in the kernel
// (fused == 2) or by the reset kernel after it (fused == 1).
int env_control_step(arc_sim* s, const float* actions, const TaskOut& O, const int* ids, int n, int* queue,
                     cudaStream_t st)
{
    const bool resets = s->fused >= 2;
    if (check(s, cudaMemsetAsync(O.done_count, 0, sizeof(int), st), "memset done_count") ||
        check(s,
              launch_control_step(s->mf, s->rm, view<float>(s), (TerrainGeom<float>*)s->tg, s->tgd, s->grid_of,
                                  s->cell, s->tp, s->ts, O, actions, static_cast<float*>(s->spill),
                                  s->spill_per_lane, s->lane_cap, ids, n, queue, resets, st),
              "control step kernel"))
        return ARC_ERR_CUDA;
    if (resets)
        return ARC_OK;
    return check(s,
                 launch_task_reset<float>(s->mf, s->rm, view<float>(s), (TerrainGeom<float>*)s->tg, s->tgd,
                                          s->grid_of, s->cell, s->tp, s->ts, s->to.obs, O.done_list, O.done_count, n,
                                          st),
                 "task reset kernel");
}

// the whole control step of ArcVecEnv.step_wait, as launched into `st`
int ensure_step_host(arc_sim* s);
bool order_applies(const arc_sim* s);
const int* range_ids(arc_sim* s, int first, int count, cudaStream_t st, int slot);

int env_step_launches(arc_sim* s, const float* actions, cudaStream_t st)
{
    // the worlds in the step order, or all worlds in index order (NULL)
    const int* ids = nullptr;
    if (order_applies(s)) {
        if (int rc = ensure_step_host(s))
            return rc;
        if (!(ids = range_ids(s, 0, s->n, st, 0)))
            return ARC_ERR_CUDA;
    }
    if (fused_applies(s))
        return env_control_step(s, actions, s->to, ids, s->n, s->use_queue ? s->queue : nullptr, st);
    Actuation A{nullptr, actions};
    int rc = step_any(s, A, st, ids, s->n);
    if (rc)
        return rc;
    rc = s->fp64 ? env_task_step<double>(s, actions, true, st) : env_task_step<float>(s, actions, true, st);
    if (rc)
        return rc;
    return s->fp64 ? env_reset_done<double>(s, st) : env_reset_done<float>(s, st);
}

constexpr int kMaxChunks = 16;

// The step kernels' world order (arc_env_set_step_order): the worlds of a
// range by difficulty band, hardest first, and by world index within a band.
// The groups of 32 worlds that the work queue hands out first are then the
// costliest, and the last, which run while the SMs empty, the cheapest
// (longest first). A world's results do not depend on which others share its
// CTA or when it runs, so any order gives the same worlds bit for bit.
constexpr int kOrderChunk = 1024;  // worlds per CTA of the two order kernels
constexpr int kOrderBands = 16;

__device__ __forceinline__ int difficulty_band(const double* __restrict__ difficulty, int w)
{
    const double d = difficulty[w];
    return d >= 1.0 ? kOrderBands - 1 : (d > 0.0 ? (int)(d * kOrderBands) : 0);  // NaN: band 0
}

// World ranges of arc_env_step_host: range c is first[c] .. first[c + 1] - 1.
struct Ranges {
    int first[kMaxChunks + 1];
};

// Ranges that halve from one to the next (rounded to 32 worlds): the copies
// of each range are shorter than the step of the next (a world's step takes
// ~3x its copies), and the last range's copies, which nothing hides, are a
// small share of all.
Ranges host_ranges(int n, int chunks)
{
    Ranges r{};
    const double total = 1.0 - std::ldexp(1.0, -chunks);
    r.first[0] = 0;
    for (int c = 1; c < chunks; ++c) {
        const double frac = (1.0 - std::ldexp(1.0, -c)) / total;
        int f = (int)std::lround(n * frac / 32.0) * 32;
        f = std::max(f, r.first[c - 1] + 1);
        r.first[c] = std::min(f, n - (chunks - c));
    }
    r.first[chunks] = n;
    return r;
}

// Ranges of near-equal size (whole 32-world groups where n allows): the
// parts of arc_env_step_part.
Ranges part_ranges(int n, int parts)
{
    Ranges r{};
    r.first[0] = 0;
    for (int c = 1; c < parts; ++c) {
        int f = (int)std::lround((double)n * c / parts / 32.0) * 32;
        f = std::max(f, r.first[c - 1] + 1);
        r.first[c] = std::min(f, n - (parts - c));
    }
    r.first[parts] = n;
    return r;
}

// The ended worlds of every range, range c's at chunk_done[first[c] ..],
// gathered into done_list in range order, and their total into done_count.
__global__ void k_merge_done(const int* __restrict__ chunk_done, const int* __restrict__ chunk_count,
                             const __grid_constant__ Ranges R, int chunks, int* __restrict__ done_list,
                             int* __restrict__ done_count)
{
    __shared__ int base[kMaxChunks + 1];
    if (threadIdx.x == 0) {
        base[0] = 0;
        for (int c = 0; c < chunks; ++c)
            base[c + 1] = base[c] + chunk_count[c];
        *done_count = base[chunks];
    }
    __syncthreads();
    for (int c = 0; c < chunks; ++c) {
        const int first = R.first[c];
        for (int k = threadIdx.x; k < chunk_count[c]; k += blockDim.x)
            done_list[base[c] + k] = chunk_done[first + k];
    }
}

// The step order of worlds first .. first + count - 1, in two launches over
// chunks of kOrderChunk worlds, one CTA each. k_order_count: each chunk's
// worlds per band into counts[chunk][band].
__global__ void __launch_bounds__(kOrderChunk) k_order_count(int* __restrict__ counts,
                                                              const double* __restrict__ difficulty, int first,
                                                              int count)
{
    __shared__ int c[kOrderBands];
    const int t = threadIdx.x, i = blockIdx.x * kOrderChunk + t;
    if (t < kOrderBands)
        c[t] = 0;
    __syncthreads();
    if (i < count)
        atomicAdd(&c[difficulty_band(difficulty, first + i)], 1);
    __syncthreads();
    if (t < kOrderBands)
        counts[blockIdx.x * kOrderBands + t] = c[t];
}

// k_order_place: each chunk's worlds to their places in order[first ..]:
// bands from the hardest, within a band the chunks in turn and each chunk's
// worlds by index (per band: a ballot per warp, then a scan over the warps).
__global__ void __launch_bounds__(kOrderChunk) k_order_place(int* __restrict__ order, const int* __restrict__ counts,
                                                              const double* __restrict__ difficulty, int first,
                                                              int count)
{
    constexpr int kWarpsPerChunk = kOrderChunk / 32;
    __shared__ int total[kOrderBands], prior[kOrderBands];  // a band's worlds: all, in the chunks before
    __shared__ int base[kOrderBands];                      // where this chunk's worlds of each band start
    __shared__ int before[kWarpsPerChunk][kOrderBands + 1];  // a band's worlds in a warp, then in the warps before
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5, chunk = blockIdx.x, i = chunk * kOrderChunk + t;
    if (warp < kOrderBands) {  // warp b sums band b over the chunks
        int all = 0, mine = 0;
        for (int k = lane; k < (int)gridDim.x; k += 32) {
            const int v = counts[k * kOrderBands + warp];
            all += v;
            mine += k < chunk ? v : 0;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            all += __shfl_xor_sync(0xffffffffu, all, o);
            mine += __shfl_xor_sync(0xffffffffu, mine, o);
        }
        if (lane == 0) {
            total[warp] = all;
            prior[warp] = mine;
        }
    }
    const int band = i < count ? difficulty_band(difficulty, first + i) : -1;
    unsigned same = 0;  // the lanes of this warp in this thread's band
#pragma unroll
    for (int b = 0; b < kOrderBands; ++b) {
        const unsigned m = __ballot_sync(0xffffffffu, band == b);
        if (lane == b)
            before[warp][b] = __popc(m);
        if (band == b)
            same = m;
    }
    __syncthreads();
    if (t == 0) {
        int at = 0;
        for (int b = kOrderBands - 1; b >= 0; --b) {
            base[b] = at + prior[b];
            at += total[b];
        }
    }
    if (warp < kOrderBands) {  // warp b: band b's exclusive scan over the chunk's warps
        const int c = before[lane][warp];
        int x = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o)
                x += y;
        }
        before[lane][warp] = x - c;
    }
    __syncthreads();
    if (band >= 0)
        order[first + base[band] + before[warp][band] + __popc(same & ((1u << lane) - 1u))] = first + i;
}

__global__ void k_iota(int* __restrict__ out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        out[i] = i;
}

int ensure_step_host(arc_sim* s)
{
    if (s->iota)
        return ARC_OK;
    // everything is made into locals and handed to s only once all of it
    // exists, so a failure part way leaves s as it was and leaks nothing
    int *iota = nullptr, *order = nullptr, *order_counts = nullptr, *chunk_done = nullptr, *chunk_count = nullptr,
        *part_queue = nullptr;
    cudaStream_t copy_in = nullptr, copy_out = nullptr;
    constexpr int kEvents = (int)(sizeof(s->ev) / sizeof(s->ev[0]));
    cudaEvent_t ev[kEvents] = {};
    auto release = [&] {
        for (cudaEvent_t e : ev)
            if (e)
                cudaEventDestroy(e);
        for (cudaStream_t c : {copy_in, copy_out})
            if (c)
                cudaStreamDestroy(c);
        for (int* p : {iota, order, order_counts, chunk_done, chunk_count, part_queue})
            cudaFree(p);
        return ARC_ERR_CUDA;
    };
    if (check(s, cudaMalloc((void**)&chunk_done, sizeof(int) * s->n), "cudaMalloc(chunk lists)") ||
        check(s, cudaMalloc((void**)&chunk_count, sizeof(int) * kMaxChunks), "cudaMalloc(chunk counts)") ||
        check(s, cudaMalloc((void**)&part_queue, sizeof(int) * 2 * kMaxChunks), "cudaMalloc(part queues)") ||
        check(s, cudaMalloc((void**)&iota, sizeof(int) * s->n), "cudaMalloc(world indices)") ||
        check(s, cudaMalloc((void**)&order, sizeof(int) * s->n), "cudaMalloc(step order)") ||
        check(s, cudaMalloc((void**)&order_counts, sizeof(int) * kOrderBands * (s->n / kOrderChunk + 2 + kMaxChunks)),
              "cudaMalloc(step order counts)"))
        return release();
    k_iota<<<(s->n + 255) / 256, 256, 0, s->stream>>>(iota, s->n);
    k_iota<<<(s->n + 255) / 256, 256, 0, s->stream>>>(order, s->n);
    // ready before any stream uses them (arc_env_step_part runs on the caller's)
    if (check(s, cudaGetLastError(), "world indices") ||
        check(s, cudaMemsetAsync(part_queue, 0, sizeof(int) * 2 * kMaxChunks, s->stream), "zero part queues") ||
        check(s, cudaStreamSynchronize(s->stream), "world indices") ||
        check(s, cudaStreamCreateWithFlags(&copy_in, cudaStreamNonBlocking), "copy stream") ||
        check(s, cudaStreamCreateWithFlags(&copy_out, cudaStreamNonBlocking), "copy stream"))
        return release();
    for (cudaEvent_t& e : ev)
        if (check(s, cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event"))
            return release();
    s->chunk_done = chunk_done;
    s->chunk_count = chunk_count;
    s->part_queue = part_queue;
    s->copy_in = copy_in;
    s->copy_out = copy_out;
    for (int i = 0; i < kEvents; ++i)
        s->ev[i] = ev[i];
    s->order = order;
    s->order_counts = order_counts;
    s->iota = iota;
    return ARC_OK;
}

// Whether the env's step kernels take the step order: on, and a kernel that
// steps lists of worlds as it steps whole batches (the leg-parallel kernel
// steps whole batches only).
bool order_applies(const arc_sim* s)
{
    return s->step_order && s->ts.difficulty && (s->kernel == ARC_KERNEL_WARPS || s->kernel == ARC_KERNEL_PLAIN);
}

// The world ids the step kernels take for worlds first .. first + count - 1:
// the range's step order, made into `st` from the worlds' current
// difficulty, when it applies; else the worlds in index order. NULL on a
// launch error. Ranges that run side by side (the parts of
// arc_env_step_part, slot = part, in world order) use disjoint parts of the
// order and of its counts: range `slot` takes the chunks from its first
// world's chunk + slot, which the next range's start cannot reach.
const int* range_ids(arc_sim* s, int first, int count, cudaStream_t st, int slot)
{
    if (!order_applies(s) || count <= 0)
        return s->iota + first;
    const int chunks = (count + kOrderChunk - 1) / kOrderChunk;
    int* counts = s->order_counts + (first / kOrderChunk + slot) * kOrderBands;
    k_order_count<<<chunks, kOrderChunk, 0, st>>>(counts, s->ts.difficulty, first, count);
    k_order_place<<<chunks, kOrderChunk, 0, st>>>(s->order, counts, s->ts.difficulty, first, count);
    if (check(s, cudaGetLastError(), "step order kernels"))
        return nullptr;
    return s->order + first;
}

// One control step of worlds first .. first + count - 1 into `st`, their
// ended worlds listed at chunk_done[first ..] with chunk_count[c] of them.
// part >= 0: a part of arc_env_step_part (its own work queue).
template <class R> int env_step_chunk(arc_sim* s, int first, int count, int c, cudaStream_t st, int part = -1)
{
    TaskOut O = s->to;
    O.done_list = s->chunk_done + first;
    O.done_count = s->chunk_count + c;
    const int* ids = range_ids(s, first, count, st, part >= 0 ? part : c);
    if (!ids)
        return ARC_ERR_CUDA;
    if (fused_applies(s)) {
        int* queue = !s->use_queue ? nullptr : (part >= 0 ? s->part_queue + 2 * part : s->queue);
        return env_control_step(s, s->actions, O, ids, count, queue, st);
    }
    Actuation A{nullptr, s->actions};
    if (int rc = step_any(s, A, st, ids, count, part))
        return rc;
    if (check(s, launch_task_step<R>(dev_model<R>(s), view<R>(s), s->tp, s->ts, O, s->actions, 2, st, first, count),
              "task step kernel") ||
        check(s, launch_task_heights<R>(dev_model<R>(s), view<R>(s), s->tp, O, st, first, count), "task heights kernel"))
        return ARC_ERR_CUDA;
    return check(s,
                 launch_task_reset<R>(dev_model<R>(s), s->rm, view<R>(s), (TerrainGeom<R>*)s->tg, s->tgd, s->grid_of,
                                      s->cell, s->tp, s->ts, s->to.obs, s->chunk_done + first, s->chunk_count + c,
                                      count, st),
                 "task reset kernel");
}

}  // namespace

extern "C" {

int arc_env_step_host(arc_sim* s, const float* h_actions, float* h_obs, float* h_reward, unsigned char* h_terminated,
                      unsigned char* h_truncated, int chunks)
{
    if (int rc = env_check(s))
        return rc;
    if (!h_actions || !h_obs)
        return fail(s, ARC_ERR_ARG, "arc_env_step_host: actions and observations are required");
    chunks = std::max(1, std::min(chunks, std::min(kMaxChunks, s->n)));
    if (int rc = ensure_step_host(s))
        return rc;
    cudaStream_t st = s->stream;
    cudaEvent_t* ev_in = s->ev;
    cudaEvent_t* ev_out = s->ev + kMaxChunks;
    cudaEvent_t ev_start = s->ev[2 * kMaxChunks], ev_end = s->ev[2 * kMaxChunks + 1];
    const Ranges R = host_ranges(s->n, chunks);
    auto range = [&](int c, int& first, int& count) {
        first = R.first[c];
        count = R.first[c + 1] - first;
    };
    // the copies start after the work already queued on the sim's stream
    if (check(s, cudaEventRecord(ev_start, st), "event") ||
        check(s, cudaStreamWaitEvent(s->copy_in, ev_start, 0), "wait") ||
        check(s, cudaStreamWaitEvent(s->copy_out, ev_start, 0), "wait") ||
        check(s, cudaMemsetAsync(s->chunk_count, 0, sizeof(int) * chunks, st), "memset counts"))
        return ARC_ERR_CUDA;
    for (int c = 0; c < chunks; ++c) {
        int first, count;
        range(c, first, count);
        if (check(s, cudaMemcpyAsync(s->actions + (size_t)first * kNumJoints, h_actions + (size_t)first * kNumJoints,
                                     sizeof(float) * kNumJoints * count, cudaMemcpyHostToDevice, s->copy_in),
                  "actions in") ||
            check(s, cudaEventRecord(ev_in[c], s->copy_in), "event"))
            return ARC_ERR_CUDA;
    }
    for (int c = 0; c < chunks; ++c) {
        int first, count;
        range(c, first, count);
        if (check(s, cudaStreamWaitEvent(st, ev_in[c], 0), "wait"))
            return ARC_ERR_CUDA;
        if (int rc = s->fp64 ? env_step_chunk<double>(s, first, count, c, st) : env_step_chunk<float>(s, first, count, c, st))
            return rc;
        if (check(s, cudaEventRecord(ev_out[c], st), "event") ||
            check(s, cudaStreamWaitEvent(s->copy_out, ev_out[c], 0), "wait") ||
            check(s, cudaMemcpyAsync(h_obs + (size_t)first * kObsSize, s->to.obs + (size_t)first * kObsSize,
                                     sizeof(float) * kObsSize * count, cudaMemcpyDeviceToHost, s->copy_out),
                  "observations out") ||
            (h_reward && check(s, cudaMemcpyAsync(h_reward + first, s->to.reward + first, sizeof(float) * count,
                                                  cudaMemcpyDeviceToHost, s->copy_out),
                               "rewards out")) ||
            (h_terminated && check(s, cudaMemcpyAsync(h_terminated + first, s->to.terminated + first, count,
                                                      cudaMemcpyDeviceToHost, s->copy_out),
                                   "terminations out")) ||
            (h_truncated && check(s, cudaMemcpyAsync(h_truncated + first, s->to.truncated + first, count,
                                                     cudaMemcpyDeviceToHost, s->copy_out),
                                  "truncations out")))
            return ARC_ERR_CUDA;
    }
    k_merge_done<<<1, 256, 0, st>>>(s->chunk_done, s->chunk_count, R, chunks, s->to.done_list, s->to.done_count);
    if (check(s, cudaGetLastError(), "merge ended worlds") || check(s, cudaEventRecord(ev_end, s->copy_out), "event") ||
        check(s, cudaStreamWaitEvent(st, ev_end, 0), "wait"))
        return ARC_ERR_CUDA;
    return sync(s, "arc_env_step_host");
}

int arc_env_part_range(const arc_sim* s, int part, int parts, int* first, int* count)
{
    if (int rc = env_check(s))
        return rc;
    if (parts < 1 || parts > std::min(kMaxChunks, s->n) || part < 0 || part >= parts)
        return fail(s, ARC_ERR_ARG, "arc_env_part_range: need 0 <= part < parts <= min(16, worlds)");
    const Ranges R = part_ranges(s->n, parts);
    if (first)
        *first = R.first[part];
    if (count)
        *count = R.first[part + 1] - R.first[part];
    return ARC_OK;
}

int arc_env_step_part(arc_sim* s, int part, int parts, void* stream)
{
    int first = 0, count = 0;
    if (int rc = arc_env_part_range(s, part, parts, &first, &count))
        return rc;
    if (int rc = ensure_step_host(s))
        return rc;
    cudaStream_t st = stream_of(s, stream);
    if (check(s, cudaMemsetAsync(s->chunk_count + part, 0, sizeof(int), st), "memset part count"))
        return ARC_ERR_CUDA;
    return s->fp64 ? env_step_chunk<double>(s, first, count, part, st, part)
                   : env_step_chunk<float>(s, first, count, part, st, part);
}

int arc_env_get_step_order(arc_sim* s, int* order)
{
    if (int rc = env_check(s))
        return rc;
    if (!order)
        return fail(s, ARC_ERR_ARG, "arc_env_get_step_order: NULL order");
    if (int rc = ensure_step_host(s))
        return rc;
    const int* ids = order_applies(s) ? range_ids(s, 0, s->n, s->stream, 0) : s->iota;
    if (!ids ||
        check(s, cudaMemcpyAsync(order, ids, sizeof(int) * s->n, cudaMemcpyDeviceToHost, s->stream), "step order"))
        return ARC_ERR_CUDA;
    return sync(s, "step order");
}

int arc_env_merge_parts(arc_sim* s, int parts, void* stream)
{
    if (int rc = arc_env_part_range(s, 0, parts, nullptr, nullptr))
        return rc;
    if (!s->iota)
        return fail(s, ARC_ERR_ARG, "arc_env_merge_parts: no part was stepped");
    cudaStream_t st = stream_of(s, stream);
    k_merge_done<<<1, 256, 0, st>>>(s->chunk_done, s->chunk_count, part_ranges(s->n, parts), parts, s->to.done_list,
                                    s->to.done_count);
    return check(s, cudaGetLastError(), "merge ended worlds");
}

int arc_env_init(arc_sim* s, const arc_task_config* cfg, unsigned long long seed)
{
    if (!s->model.leaper)
        return fail(s, ARC_ERR_UNSUPPORTED, "the task layer needs the quadruped model");
    if (s->env)
        return ARC_OK;
    arc_task_config c;
    if (cfg)
        c = *cfg;
    else
        arc_task_config_default(&c);
    TaskParams& P = s->tp;
    std::memset(&P, 0, sizeof(P));
    P.dt = c.dt;
    P.max_steps = c.max_steps;
    P.action_scale = c.action_scale;
    P.checkpoint_radius = c.checkpoint_radius;
    P.checkpoint_min_dist = c.checkpoint_min_dist;
    P.checkpoint_max_dist = c.checkpoint_max_dist;
    P.border = c.border;
    P.w_progress = c.w_progress;
    P.max_speed = c.max_speed;
    P.fov = c.fov;
    P.w_turn = c.w_turn;
    P.w_checkpoint = c.w_checkpoint;
    P.w_time = c.w_time;
    P.w_fall = c.w_fall;
    P.w_energy = c.w_energy;
    P.w_action_rate = c.w_action_rate;
    P.w_body_contact = c.w_body_contact;
    P.w_torso_contact = c.w_torso_contact;
    P.w_body_rate = c.w_body_rate;
    P.w_bounce = c.w_bounce;
    P.flip_up_z = c.flip_up_z;
    P.beached_steps = c.beached_steps;
    P.void_z = c.void_z;
    P.curriculum = c.curriculum;
    P.difficulty = c.difficulty;
    P.max_difficulty = c.max_difficulty;
    P.level_step = c.level_step;
    P.level_up_checkpoints = c.level_up_checkpoints;
    P.level_down_steps = c.level_down_steps;
    P.fov_rad = c.fov * (kPi / 180.0);  // np.radians multiplies by pi/180
    P.cos_fov = std::cos(P.fov_rad);
    P.half_extent = 0.5 * s->grid * s->cell;
    P.stand_height = s->model.stand_height;
    for (int j = 0; j < kNumJoints; ++j)
        P.default_angles[j] = s->model.default_angles[j];
    // arc/task.py:74-76: np.arange(-1.0, 1.41, 0.2) x np.arange(-1.0, 1.01, 0.2)
    int k = 0;
    for (int a = 0; a < 13; ++a)
        for (int b = 0; b < 11; ++b, ++k) {
            P.offsets[k][0] = -1.0 + a * 0.2;
            P.offsets[k][1] = -1.0 + b * 0.2;
        }
    P.seed = seed;
    // the action scale of the actuation follows the task config
    s->mf.action_scale = c.action_scale;
    s->md.action_scale = c.action_scale;

    const size_t n = (size_t)std::max(s->n, 1);
    bool ok = true;
    TaskState& S = s->ts;
    S.target = env_alloc<double>(s, 2 * n, ok);
    S.target_z = env_alloc<double>(s, n, ok);
    S.prev_dist = env_alloc<double>(s, n, ok);
    S.prev_gaze = env_alloc<double>(s, n, ok);
    S.prev_action = env_alloc<float>(s, n * kNumJoints, ok);
    S.torso_steps = env_alloc<int>(s, n, ok);
    S.steps = env_alloc<int>(s, n, ok);
    S.checkpoints = env_alloc<int>(s, n, ok);
    S.level = env_alloc<double>(s, n, ok);
    S.difficulty = env_alloc<double>(s, n, ok);
    S.in_view = env_alloc<unsigned char>(s, n, ok);
    S.episode = env_alloc<unsigned>(s, n, ok);
    S.draws = env_alloc<unsigned>(s, n, ok);
    TaskOut& O = s->to;
    O.obs = env_alloc<float>(s, n * kObsSize, ok);
    O.terminal_obs = env_alloc<float>(s, n * kObsSize, ok);
    O.reward = env_alloc<float>(s, n, ok);
    O.terminated = env_alloc<unsigned char>(s, n, ok);
    O.truncated = env_alloc<unsigned char>(s, n, ok);
    O.cause = env_alloc<signed char>(s, n, ok);
    O.ended_checkpoints = env_alloc<int>(s, n, ok);
    O.ended_difficulty = env_alloc<double>(s, n, ok);
    O.ended_steps = env_alloc<int>(s, n, ok);
    O.done_list = env_alloc<int>(s, n, ok);
    O.done_count = env_alloc<int>(s, 1, ok);
    s->actions = env_alloc<float>(s, n * kNumJoints, ok);
    if (!ok)
        return fail(s, ARC_ERR_CUDA, "arc_env_init: device allocation failed");
    // initial level / difficulty (arc/task.py:107-108)
    std::vector<double> lvl(n, c.curriculum ? 0.0 : c.difficulty);
    if (check(s, cudaMemcpy(S.level, lvl.data(), n * sizeof(double), cudaMemcpyHostToDevice), "level") ||
        check(s, cudaMemcpy(S.difficulty, lvl.data(), n * sizeof(double), cudaMemcpyHostToDevice), "difficulty") ||
        // the buffers' zeroing (legacy default stream) before any kernel on the sim's stream
        check(s, cudaDeviceSynchronize(), "env init"))
        return ARC_ERR_CUDA;
    s->env = true;
    return ARC_OK;
}

int arc_env_reset(arc_sim* s, const int* ids, int n_ids, void* stream)
{
    if (int rc = env_check(s))
        return rc;
    cudaStream_t st = stream_of(s, stream);
    std::vector<int> all;
    if (!ids || n_ids < 0) {
        all.resize(s->n);
        for (int i = 0; i < s->n; ++i)
            all[i] = i;
        ids = all.data();
        n_ids = s->n;
    }
    if (n_ids == 0)
        return ARC_OK;
    if (!ids_ok(s, ids, n_ids))
        return fail(s, ARC_ERR_ARG, "arc_env_reset: world index out of range");
    int* d = (int*)grow(s, s->st_in3, sizeof(int) * n_ids);
    if (!d)
        return ARC_ERR_CUDA;
    if (check(s, cudaMemcpyAsync(d, ids, sizeof(int) * n_ids, cudaMemcpyHostToDevice, st), "reset ids"))
        return ARC_ERR_CUDA;
    cudaError_t e =
        s->fp64 ? launch_task_reset<double>(s->md, s->rm, view<double>(s), (TerrainGeom<double>*)s->tg, s->tgd,
                                            s->grid_of, s->cell, s->tp, s->ts, s->to.obs, d, nullptr, n_ids, st)
                : launch_task_reset<float>(s->mf, s->rm, view<float>(s), (TerrainGeom<float>*)s->tg, s->tgd,
                                           s->grid_of, s->cell, s->tp, s->ts, s->to.obs, d, nullptr, n_ids, st);
    if (check(s, e, "task reset kernel"))
        return ARC_ERR_CUDA;
    return check(s, cudaStreamSynchronize(st), "arc_env_reset");
}

int arc_env_admit(arc_sim* s, const int* ids, int n_ids, const double* difficulty, const unsigned* keys, void* stream)
{
    if (int rc = env_check(s))
        return rc;
    if (n_ids < 0 || (n_ids > 0 && (!ids || !difficulty || !keys)))
        return fail(s, ARC_ERR_ARG, "arc_env_admit: bad arguments");
    if (n_ids == 0)
        return ARC_OK;
    if (!ids_ok(s, ids, n_ids))
        return fail(s, ARC_ERR_ARG, "arc_env_admit: world index out of range");
    cudaStream_t st = stream_of(s, stream);
    if (!s->ts.key) {
        // every world keeps its index as its key until a tenant gives it one
        bool ok = true;
        unsigned* key = env_alloc<unsigned>(s, (size_t)s->n, ok);
        if (!ok)
            return fail(s, ARC_ERR_CUDA, "arc_env_admit: device allocation failed");
        k_iota<<<(s->n + 255) / 256, 256, 0, st>>>(reinterpret_cast<int*>(key), s->n);
        if (check(s, cudaGetLastError(), "world keys"))
            return ARC_ERR_CUDA;
        s->ts.key = key;
    }
    const size_t n = (size_t)n_ids;
    unsigned char* d = (unsigned char*)grow(s, s->st_in3, n * (sizeof(int) + sizeof(double) + sizeof(unsigned)));
    if (!d)
        return ARC_ERR_CUDA;
    double* d_diff = reinterpret_cast<double*>(d);
    int* d_ids = reinterpret_cast<int*>(d + n * sizeof(double));
    unsigned* d_keys = reinterpret_cast<unsigned*>(d + n * (sizeof(double) + sizeof(int)));
    if (check(s, cudaMemcpyAsync(d_diff, difficulty, n * sizeof(double), cudaMemcpyHostToDevice, st), "admit") ||
        check(s, cudaMemcpyAsync(d_ids, ids, n * sizeof(int), cudaMemcpyHostToDevice, st), "admit") ||
        check(s, cudaMemcpyAsync(d_keys, keys, n * sizeof(unsigned), cudaMemcpyHostToDevice, st), "admit"))
        return ARC_ERR_CUDA;
    cudaError_t e =
        s->fp64 ? launch_env_admit<double>(s->md, s->rm, view<double>(s), (TerrainGeom<double>*)s->tg, s->tgd,
                                           s->grid_of, s->cell, s->tp, s->ts, s->to.obs, d_ids, d_diff, d_keys,
                                           n_ids, st)
                : launch_env_admit<float>(s->mf, s->rm, view<float>(s), (TerrainGeom<float>*)s->tg, s->tgd,
                                          s->grid_of, s->cell, s->tp, s->ts, s->to.obs, d_ids, d_diff, d_keys,
                                          n_ids, st);
    if (check(s, e, "admit kernels"))
        return ARC_ERR_CUDA;
    return check(s, cudaStreamSynchronize(st), "arc_env_admit");
}

int arc_env_step_ids(arc_sim* s, const int* d_ids, int n_ids, void* stream)
{
    if (int rc = env_check(s))
        return rc;
    if (n_ids < 0 || (n_ids > 0 && !d_ids))
        return fail(s, ARC_ERR_ARG, "arc_env_step_ids: bad arguments");
    if (n_ids == 0)
        return ARC_OK;
    cudaStream_t st = stream_of(s, stream);
    if (fused_applies(s))
        return env_control_step(s, s->actions, s->to, d_ids, n_ids, s->use_queue ? s->queue : nullptr, st);
    Actuation A{nullptr, s->actions};
    if (int rc = step_any(s, A, st, d_ids, n_ids))
        return rc;
    if (check(s, cudaMemsetAsync(s->to.done_count, 0, sizeof(int), st), "memset done_count"))
        return ARC_ERR_CUDA;
    cudaError_t e = s->fp64 ? launch_task_step<double>(s->md, view<double>(s), s->tp, s->ts, s->to, s->actions, 2, st,
                                                       0, n_ids, d_ids)
                            : launch_task_step<float>(s->mf, view<float>(s), s->tp, s->ts, s->to, s->actions, 2, st,
                                                      0, n_ids, d_ids);
    if (check(s, e, "task step kernel"))
        return ARC_ERR_CUDA;
    e = s->fp64 ? launch_task_heights<double>(s->md, view<double>(s), s->tp, s->to, st, 0, n_ids, d_ids)
                : launch_task_heights<float>(s->mf, view<float>(s), s->tp, s->to, st, 0, n_ids, d_ids);
    if (check(s, e, "task heights kernel"))
        return ARC_ERR_CUDA;
    return s->fp64 ? env_reset_done<double>(s, st) : env_reset_done<float>(s, st);
}

int arc_env_step(arc_sim* s, const float* d_actions, void* stream)
{
    if (int rc = env_check(s))
        return rc;
    cudaStream_t st = stream_of(s, stream);
    if (d_actions)
        return env_step_launches(s, d_actions, st);
    // graph of the whole control step over the ARC_ENV_ACTIONS buffer
    if (s->graph_exec && (s->graph_kernel != s->kernel || s->graph_wpc != s->wpc ||
                          s->graph_queue != (int)s->use_queue || s->graph_fused != s->fused ||
                          s->graph_tile != s->substep_tile || s->graph_lastc != s->lastc ||
                          s->graph_order != s->step_order)) {
        cudaGraphExecDestroy(s->graph_exec);
        cudaGraphDestroy(s->graph);
        s->graph_exec = nullptr;
        s->graph = nullptr;
    }
    if (!s->graph_exec) {
        // one eager step first: kernels configure their attributes outside capture
        // (this step is real work on the current actions, like every other step)
        if (int rc = env_step_launches(s, s->actions, st))
            return rc;
        if (!s->graph_stream &&
            check(s, cudaStreamCreateWithFlags(&s->graph_stream, cudaStreamNonBlocking), "graph stream"))
            return ARC_ERR_CUDA;
        if (check(s, cudaStreamSynchronize(st), "pre-capture sync") ||
            check(s, cudaStreamBeginCapture(s->graph_stream, cudaStreamCaptureModeThreadLocal), "begin capture"))
            return ARC_ERR_CUDA;
        int rc = env_step_launches(s, s->actions, s->graph_stream);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(s->graph_stream, &g);
        if (rc)
            return rc;
        if (check(s, e, "end capture") || check(s, cudaGraphInstantiate(&s->graph_exec, g, 0), "instantiate"))
            return ARC_ERR_CUDA;
        s->graph = g;
        s->graph_kernel = s->kernel;
        s->graph_wpc = s->wpc;
        s->graph_queue = (int)s->use_queue;
        s->graph_fused = s->fused;
        s->graph_tile = s->substep_tile;
        s->graph_lastc = s->lastc;
        s->graph_order = s->step_order;
        return ARC_OK;
    }
    return check(s, cudaGraphLaunch(s->graph_exec, st), "graph launch");
}

int arc_env_task_step(arc_sim* s, const float* d_actions, void* stream)
{
    if (int rc = env_check(s))
        return rc;
    cudaStream_t st = stream_of(s, stream);
    const float* a = d_actions ? d_actions : s->actions;
    Actuation A{nullptr, a};
    if (int rc = step_any(s, A, st))
        return rc;
    return s->fp64 ? env_task_step<double>(s, a, false, st) : env_task_step<float>(s, a, false, st);
}

int arc_env_observe(arc_sim* s, void* stream)
{
    if (int rc = env_check(s))
        return rc;
    cudaStream_t st = stream_of(s, stream);
    cudaError_t e = s->fp64 ? launch_task_observe<double>(s->md, view<double>(s), s->tp, s->ts, s->to.obs, nullptr,
                                                          s->n, st)
                            : launch_task_observe<float>(s->mf, view<float>(s), s->tp, s->ts, s->to.obs, nullptr,
                                                         s->n, st);
    return check(s, e, "task observe kernel");
}

int arc_env_buffer(const arc_sim* s, int which, void** ptr, long long* shape, int* ndim, int* code, int* bits)
{
    if (int rc = env_check(s))
        return rc;
    const long long n = s->n;
    void* p = nullptr;
    long long sh[2] = {n, 1};
    int nd = 1, c = 2, b = 32;
    switch (which) {
    case ARC_ENV_OBS: p = s->to.obs; sh[1] = kObsSize; nd = 2; break;
    case ARC_ENV_TERMINAL_OBS: p = s->to.terminal_obs; sh[1] = kObsSize; nd = 2; break;
    case ARC_ENV_REWARD: p = s->to.reward; break;
    case ARC_ENV_TERMINATED: p = s->to.terminated; c = 1; b = 8; break;
    case ARC_ENV_TRUNCATED: p = s->to.truncated; c = 1; b = 8; break;
    case ARC_ENV_CAUSE: p = s->to.cause; c = 0; b = 8; break;
    case ARC_ENV_DONE_LIST: p = s->to.done_list; c = 0; break;
    case ARC_ENV_DONE_COUNT: p = s->to.done_count; c = 0; sh[0] = 1; break;
    case ARC_ENV_ACTIONS: p = s->actions; sh[1] = kNumJoints; nd = 2; break;
    case ARC_ENV_ENDED_CHECKPOINTS: p = s->to.ended_checkpoints; c = 0; break;
    case ARC_ENV_ENDED_STEPS: p = s->to.ended_steps; c = 0; break;
    case ARC_ENV_ENDED_DIFFICULTY: p = s->to.ended_difficulty; b = 64; break;
    default: return fail(s, ARC_ERR_ARG, "arc_env_buffer: unknown buffer");
    }
    if (ptr)
        *ptr = p;
    if (shape) {
        shape[0] = sh[0];
        shape[1] = sh[1];
    }
    if (ndim)
        *ndim = nd;
    if (code)
        *code = c;
    if (bits)
        *bits = b;
    return ARC_OK;
}

}  // extern "C"

namespace {

// DLPack v0.8 ABI (dlpack.h): the exchange format torch.from_dlpack reads.
struct DLDevice_ {
    int32_t device_type;  // kDLCUDA = 2
    int32_t device_id;
};
struct DLDataType_ {
    uint8_t code, bits;
    uint16_t lanes;
};
struct DLTensor_ {
    void* data;
    DLDevice_ device;
    int32_t ndim;
    DLDataType_ dtype;
    int64_t* shape;
    int64_t* strides;
    uint64_t byte_offset;
};
struct DLManagedTensor_ {
    DLTensor_ dl_tensor;
    void* manager_ctx;
    void (*deleter)(DLManagedTensor_*);
};
struct DLPackHolder {
    DLManagedTensor_ t;
    int64_t shape[2];
};

void dlpack_delete(DLManagedTensor_* t) { delete reinterpret_cast<DLPackHolder*>(t->manager_ctx); }

}  // namespace

extern "C" {

int arc_env_dlpack(const arc_sim* s, int which, void** managed)
{
    void* p;
    long long shape[2];
    int nd, code, bits;
    if (int rc = arc_env_buffer(s, which, &p, shape, &nd, &code, &bits))
        return rc;
    int dev = 0;
    cudaGetDevice(&dev);
    DLPackHolder* h = new DLPackHolder();
    h->shape[0] = shape[0];
    h->shape[1] = shape[1];
    h->t.dl_tensor.data = p;
    h->t.dl_tensor.device = DLDevice_{2, dev};
    h->t.dl_tensor.ndim = nd;
    h->t.dl_tensor.dtype = DLDataType_{(uint8_t)code, (uint8_t)bits, 1};
    h->t.dl_tensor.shape = h->shape;
    h->t.dl_tensor.strides = nullptr;  // compact row-major
    h->t.dl_tensor.byte_offset = 0;
    h->t.manager_ctx = h;
    h->t.deleter = dlpack_delete;
    *managed = &h->t;
    return ARC_OK;
}

static int env_copy(const arc_sim* s, int which, void* host, bool down)
{
    void* p;
    long long shape[2];
    int nd, code, bits;
    if (int rc = arc_env_buffer(s, which, &p, shape, &nd, &code, &bits))
        return rc;
    const size_t bytes = (size_t)shape[0] * (nd == 2 ? shape[1] : 1) * (bits / 8);
    if (sync(s, "env copy"))
        return ARC_ERR_CUDA;
    return check(s, cudaMemcpy(down ? host : p, down ? p : host, bytes,
                               down ? cudaMemcpyDeviceToHost : cudaMemcpyHostToDevice),
                 "env copy");
}

int arc_env_download(const arc_sim* s, int which, void* host) { return env_copy(s, which, host, true); }
int arc_env_upload(arc_sim* s, int which, const void* host) { return env_copy(s, which, (void*)host, false); }

int arc_env_get_task_state(const arc_sim* s, const int* ids, int n_ids, double* out)
{
    if (int rc = env_check(s))
        return rc;
    if (!ids_ok(s, ids, n_ids))
        return fail(s, ARC_ERR_ARG, "arc_env_get_task_state: world index out of range");
    if (sync(s, "task state"))
        return ARC_ERR_CUDA;
    const size_t n = s->n;
    std::vector<double> tgt(2 * n), tz(n), pd(n), pg(n), lvl(n), dif(n);
    std::vector<float> pa(n * kNumJoints);
    std::vector<int> ts(n), st(n), cp(n);
    std::vector<unsigned char> iv(n);
    std::vector<unsigned> ep(n), dr(n);
    const TaskState& S = s->ts;
    bool ok = cudaMemcpy(tgt.data(), S.target, 2 * n * 8, cudaMemcpyDeviceToHost) == cudaSuccess &&
              cudaMemcpy(tz.data(), S.target_z, n * 8, cudaMemcpyDeviceToHost) == cudaSuccess &&
              cudaMemcpy(pd.data(), S.prev_dist, n * 8, cudaMemcpyDeviceToHost) == cudaSuccess &&
              cudaMemcpy(pg.data(), S.prev_gaze, n * 8, cudaMemcpyDeviceToHost) == cudaSuccess &&
              cudaMemcpy(pa.data(), S.prev_action, n * kNumJoints * 4, cudaMemcpyDeviceToHost) == cudaSuccess &&
              cudaMemcpy(ts.data(), S.torso_steps, n * 4, cudaMemcpyDeviceToHost) == cudaSuccess &&
              cudaMemcpy(st.data(), S.steps, n * 4, cudaMemcpyDeviceToHost) == cudaSuccess &&
              cudaMemcpy(cp.data(), S.checkpoints, n * 4, cudaMemcpyDeviceToHost) == cudaSuccess &&
              cudaMemcpy(lvl.data(), S.level, n * 8, cudaMemcpyDeviceToHost) == cudaSuccess &&
              cudaMemcpy(dif.data(), S.difficulty, n * 8, cudaMemcpyDeviceToHost) == cudaSuccess &&
              cudaMemcpy(iv.data(), S.in_view, n, cudaMemcpyDeviceToHost) == cudaSuccess &&
              cudaMemcpy(ep.data(), S.episode, n * 4, cudaMemcpyDeviceToHost) == cudaSuccess &&
              cudaMemcpy(dr.data(), S.draws, n * 4, cudaMemcpyDeviceToHost) == cudaSuccess;
    if (!ok)
        return check(s, cudaGetLastError(), "task state copy");
    for (int k = 0; k < n_ids; ++k) {
        const int i = ids[k];
        double* o = out + (size_t)k * ARC_TASK_STATE_SIZE;
        o[0] = tgt[2 * i];
        o[1] = tgt[2 * i + 1];
        o[2] = tz[i];
        o[3] = pd[i];
        o[4] = pg[i];
        for (int j = 0; j < kNumJoints; ++j)
            o[5 + j] = pa[(size_t)i * kNumJoints + j];
        o[17] = ts[i];
        o[18] = st[i];
        o[19] = cp[i];
        o[20] = lvl[i];
        o[21] = dif[i];
        o[22] = iv[i];
        o[23] = ep[i];
        o[24] = dr[i];
    }
    return ARC_OK;
}

int arc_env_set_task_state(arc_sim* s, const int* ids, int n_ids, const double* in)
{
    if (int rc = env_check(s))
        return rc;
    if (!ids_ok(s, ids, n_ids))
        return fail(s, ARC_ERR_ARG, "arc_env_set_task_state: world index out of range");
    if (sync(s, "task state"))
        return ARC_ERR_CUDA;
    const TaskState& S = s->ts;
    for (int k = 0; k < n_ids; ++k) {
        const int i = ids[k];
        const double* p = in + (size_t)k * ARC_TASK_STATE_SIZE;
        float pa[kNumJoints];
        for (int j = 0; j < kNumJoints; ++j)
            pa[j] = (float)p[5 + j];
        int ints[3] = {(int)p[17], (int)p[18], (int)p[19]};
        unsigned char iv = p[22] != 0.0;
        unsigned ep = (unsigned)p[23], dr = (unsigned)p[24];
        bool ok = cudaMemcpy(S.target + 2 * i, p, 16, cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(S.target_z + i, p + 2, 8, cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(S.prev_dist + i, p + 3, 8, cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(S.prev_gaze + i, p + 4, 8, cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(S.prev_action + (size_t)i * kNumJoints, pa, sizeof(pa), cudaMemcpyHostToDevice) ==
                      cudaSuccess &&
                  cudaMemcpy(S.torso_steps + i, &ints[0], 4, cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(S.steps + i, &ints[1], 4, cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(S.checkpoints + i, &ints[2], 4, cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(S.level + i, p + 20, 8, cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(S.difficulty + i, p + 21, 8, cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(S.in_view + i, &iv, 1, cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(S.episode + i, &ep, 4, cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(S.draws + i, &dr, 4, cudaMemcpyHostToDevice) == cudaSuccess;
        if (!ok)
            return check(s, cudaGetLastError(), "task state copy");
    }
    return ARC_OK;
}

int arc_env_set_targets(arc_sim* s, const int* ids, int n_ids, const double* xy)
{
    if (int rc = env_check(s))
        return rc;
    if (n_ids <= 0)
        return ARC_OK;
    if (!ids_ok(s, ids, n_ids))
        return fail(s, ARC_ERR_ARG, "arc_env_set_targets: world index out of range");
    char* buf = (char*)grow(s, s->st_in3, (size_t)n_ids * (2 * sizeof(double) + sizeof(int)));
    if (!buf)
        return ARC_ERR_CUDA;
    double* dxy = (double*)buf;
    int* dids = (int*)(buf + (size_t)n_ids * 2 * sizeof(double));
    if (check(s, cudaMemcpyAsync(dxy, xy, sizeof(double) * 2 * n_ids, cudaMemcpyHostToDevice, s->stream), "xy") ||
        check(s, cudaMemcpyAsync(dids, ids, sizeof(int) * n_ids, cudaMemcpyHostToDevice, s->stream), "ids"))
        return ARC_ERR_CUDA;
    cudaError_t e = s->fp64 ? launch_task_set_targets<double>(view<double>(s), s->tp, s->ts, dids, dxy, n_ids, s->stream)
                            : launch_task_set_targets<float>(view<float>(s), s->tp, s->ts, dids, dxy, n_ids, s->stream);
    if (check(s, e, "set targets kernel"))
        return ARC_ERR_CUDA;
    return sync(s, "arc_env_set_targets");
}

}  // extern "C"

SimView arc::sim_view(const arc_sim* s)
{
    return SimView{&s->model, view<float>(s), view<double>(s), s->fp64, s->n, s->stream};
}

bool arc::sim_task_view(const arc_sim* s, TaskState* state, double* checkpoint_radius)
{
    if (!s || !s->env)
        return false;
    *state = s->ts;
    *checkpoint_radius = s->tp.checkpoint_radius;
    return true;
}
