// Serving runtime: a continuous-batching request loop for anneal-and-certify
// jobs on one GPU.
//
//   submit   copies a job into the queue (no device work);
//   step     one round of the loop:
//              admit queued jobs while a job slot is free and the job's state
//              (R*n replica squares + quench scratch + FP64 best) fits the HBM
//              arena (first fit, looking past up to 16 jobs that do not fit yet);
//              collect the slices that have finished;
//              start the next anneal slice of every idle job, one launch per
//              cluster shape, each launch a cohort on its own stream -- jobs
//              admitted at different times, at different sweep counts, run side
//              by side, their state resident in HBM between slices, and no
//              cohort waits for another (no barrier across the GPU per round);
//              hand the jobs whose budget ran out to the retirement thread,
//              which polishes, certifies and retires them on a stream of the
//              highest priority while the cohorts anneal, and gives their slot
//              and arena space to the next;
//   poll     hands back a finished job's result and best packing.
// A job's result is the same here as alone through sqs_anneal_batch: its
// trajectory depends on its inputs and seed only.
//
// Reference: campaigns run one search process per n (scheduler.run_gpu,
// cuda/scheduler.py:80-89) with at most four concurrent workers admitted by
// free VRAM and RAM (cpp_loop.concurrency, cuda/cpp_loop.py:41-45) and a
// device-to-host synchronisation after every epoch (seeded.cu:919).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <condition_variable>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "anneal_host.h"

using namespace sqs;
using namespace sqs::ann;

namespace {

enum JobState { kQueued = 0, kActive = 1, kDone = 2 };

struct SJob {
    int64_t id = 0;
    int state = kQueued;
    int slot = -1;
    bool cancel = false;
    sqs_job job{};
    std::vector<double> xya, xya_rep;  // copies of the initial state(s)
    JobDev jd{};
    JobMut jm{};
    Plan plan{};
    int64_t left = 0;           // sweeps not yet launched
    size_t off = 0, bytes = 0;  // arena block
    sqs_job_result res{};
    std::vector<double> best;   // certified packing (n x 3) when done
};

}  // namespace

namespace {
// One in-flight slice: the jobs of one cluster shape, launched on the
// cohort's own stream and finished independently of the other cohorts.
struct Cohort {
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    int32_t* d_list = nullptr;    // the cohort's job slots (device)
    int32_t* d_status = nullptr;  // their status after the slice (device)
    int32_t* h_status = nullptr;  // ... and its pinned host copy
    std::vector<int32_t> slots;
    bool busy = false;
};
constexpr int kCohorts = 8;
constexpr double kWaitSeconds = 2e-3;
// Retirement threads.  One: several threads issuing CUDA calls at once
// slowed every phase (measured: a stream of 480 jobs at 1,000/s took 2.2 s
// with three against 0.77 s with one).
constexpr int kRetirers = 1;
// Device buffers of a retirement thread's context, reserved up front (about
// 420 bytes per square of a retired batch for the certifier's staging, the
// interval cache of its undecided squares, the rescue polish's state).
constexpr size_t kRetireStaging = (size_t)64 << 20;
constexpr size_t kRetireCache = (size_t)32 << 20;
constexpr size_t kRetirePolish = (size_t)8 << 20;
constexpr size_t kRetireHost = (size_t)8 << 20;  // pinned literal slice tables

// A retirement thread's own context (buffers, a stream of the highest
// priority) and device list of job slots.
struct Retirer {
    sqs_ctx* ctx = nullptr;
    int32_t* d_list = nullptr;
    std::thread th;
};
}  // namespace

struct sqs_server {
    sqs_ctx* ctx = nullptr;
    char* arena = nullptr;
    size_t arena_bytes = 0;
    std::map<size_t, size_t> free_blocks;  // offset -> bytes
    int max_active = 0, slice = 0;  // slice < 0: about -slice proposals per replica per step, per job
    JobDev* d_jd = nullptr;
    JobMut* d_jm = nullptr;
    std::vector<int64_t> slot_job;         // job id per slot, -1 free
    std::deque<int64_t> queue;
    std::unordered_map<int64_t, SJob> jobs;
    int64_t next_id = 1;
    std::vector<uint8_t> flying;           // per slot: in a cohort's slice now
    std::vector<uint8_t> retiring;         // per slot: handed to the retirement thread
    std::vector<Cohort> cohorts;
    // Admission uploads and builds job state on its own stream of the
    // highest priority; every slice launch waits for its last event on the
    // device, so admission needs no host synchronisation.
    cudaStream_t ast = nullptr;
    cudaEvent_t admitted = nullptr;
    // The retirement thread and what it shares with the caller's thread
    // (jobs, slots, arena, counters), guarded by `mu`.
    std::mutex mu;
    std::condition_variable cv;
    std::deque<std::vector<int32_t>> rq;   // batches of finished slots, in order
    int64_t retire_pending = 0;            // batches queued or being retired
    bool stop = false;
    int werr = 0;
    std::string werr_msg;
    std::vector<Retirer> retirers;
    size_t used = 0;
    sqs_server_stats st{};
};

namespace {

size_t arena_alloc(sqs_server* s, size_t bytes) {
    for (auto it = s->free_blocks.begin(); it != s->free_blocks.end(); ++it) {
        if (it->second < bytes) continue;
        const size_t off = it->first, rest = it->second - bytes;
        s->free_blocks.erase(it);
        if (rest) s->free_blocks[off + bytes] = rest;
        s->used += bytes;
        return off;
    }
    return (size_t)-1;
}

void arena_free(sqs_server* s, size_t off, size_t bytes) {
    s->used -= bytes;
    auto nx = s->free_blocks.lower_bound(off);
    if (nx != s->free_blocks.end() && off + bytes == nx->first) {
        bytes += nx->second;
        nx = s->free_blocks.erase(nx);
    }
    if (nx != s->free_blocks.begin()) {
        auto pv = std::prev(nx);
        if (pv->first + pv->second == off) {
            pv->second += bytes;
            return;
        }
    }
    s->free_blocks[off] = bytes;
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Every replica of a job starts from its state xya (n x 3 doubles, staged in
// the job's best-packing slot): centres as floats, angles reduced to
// [0, pi/2) in double first -- the host's init_replicas, bit for bit (fmod is
// exact, the conversions round to nearest) -- and the quench scratch zeroed.
__global__ void init_replicas_kernel(const double* __restrict__ xya, int n, int R, float4* __restrict__ dst) {
    const int64_t total = (int64_t)R * n * (1 + kQuenchScr);
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
        if (k >= (int64_t)R * n) {
            dst[k] = make_float4(0.f, 0.f, 0.f, 0.f);
            continue;
        }
        const int i = (int)(k % n);
        const double q = 1.57079632679489661923;
        double a = fmod(xya[3 * i + 2], q);
        if (a < 0.0) a += q;
        dst[k] = make_float4((float)xya[3 * i], (float)xya[3 * i + 1], (float)a, 0.f);
    }
}

size_t job_bytes(const sqs_job& J) {
    const size_t b = sizeof(float4) * (size_t)job_pos_elems(J) + sizeof(double) * 3 * (size_t)J.n;
    return (b + 255) & ~(size_t)255;
}

int admit(sqs_server* s) {
    const size_t window = 16;  // queued jobs that do not fit yet which admission looks past
    size_t skipped = 0;
    int slot = 0;
    std::vector<std::vector<float4>> inits;  // host staging of jobs with one start per replica
    bool admitted_any = false;
    for (auto it = s->queue.begin(); it != s->queue.end() && skipped < window;) {
        SJob& j = s->jobs[*it];
        while (slot < s->max_active && s->slot_job[(size_t)slot] >= 0) ++slot;
        if (slot >= s->max_active) break;
        const size_t bytes = job_bytes(j.job);
        const size_t off = arena_alloc(s, bytes);
        if (off == (size_t)-1) {
            ++skipped;
            ++it;
            continue;
        }
        j.off = off;
        j.bytes = bytes;
        j.slot = slot;
        j.state = kActive;
        j.jd.pos_off = (int64_t)(off / sizeof(float4));
        j.jd.scr_off = j.jd.pos_off + (int64_t)j.job.replicas * j.job.n;
        j.jd.best_off = (int64_t)((off + sizeof(float4) * (size_t)job_pos_elems(j.job)) / sizeof(double));
        if (s->slice < 0) {  // this job's sweeps per step: about -slice proposals, whole exchange intervals
            const int xe = std::max(1, j.jd.exchange_every);
            const int64_t sw = std::max<int64_t>(1, (-(int64_t)s->slice + j.job.n - 1) / j.job.n);
            j.jd.slice = (int)std::min<int64_t>((sw + xe - 1) / xe * xe, 1 << 30);
        }
        if (j.job.xya_rep) {  // one start per replica: built on the host
            inits.emplace_back((size_t)job_pos_elems(j.job), make_float4(0.f, 0.f, 0.f, 0.f));
            std::vector<float4>& init = inits.back();
            init_replicas(j.job, init.data());
            SQS_CUDA(cudaMemcpyAsync(s->arena + off, init.data(), sizeof(float4) * init.size(),
                                     cudaMemcpyHostToDevice, s->ast));
        } else {  // one start for all: n x 3 doubles up, replicas built on the device
            double* stage = (double*)s->arena + j.jd.best_off;
            SQS_CUDA(cudaMemcpyAsync(stage, j.xya.data(), sizeof(double) * 3 * (size_t)j.job.n,
                                     cudaMemcpyHostToDevice, s->ast));
            const int64_t total = job_pos_elems(j.job);
            const int blocks = (int)std::min<int64_t>(1024, (total + 255) / 256);
            init_replicas_kernel<<<blocks, 256, 0, s->ast>>>(stage, j.job.n, j.job.replicas,
                                                                     (float4*)(s->arena + off));
            SQS_CUDA(cudaGetLastError());
            s->ctx->launches += 1;
        }
        SQS_CUDA(cudaMemcpyAsync(s->d_jd + slot, &j.jd, sizeof(JobDev), cudaMemcpyHostToDevice, s->ast));
        SQS_CUDA(cudaMemcpyAsync(s->d_jm + slot, &j.jm, sizeof(JobMut), cudaMemcpyHostToDevice, s->ast));
        s->slot_job[(size_t)slot] = j.id;
        admitted_any = true;
        ++s->st.admitted;
        it = s->queue.erase(it);
    }
    // (copies from pageable memory have consumed their host source on return,
    // so the staging vectors may end here)
    if (admitted_any) SQS_CUDA(cudaEventRecord(s->admitted, s->ast));
    return SQS_OK;
}

}  // namespace

namespace {
void retire_loop(sqs_server* s, Retirer* me);

// Release everything a server holds (after its streams are idle).
void free_server(sqs_server* s) {
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    for (Retirer& w : s->retirers)
        if (w.th.joinable()) w.th.join();
    if (s->ast) cudaStreamSynchronize(s->ast);
    for (Cohort& c : s->cohorts) {
        if (c.st) cudaStreamSynchronize(c.st);
        if (c.st) cudaStreamDestroy(c.st);
        if (c.done) cudaEventDestroy(c.done);
        cudaFree(c.d_list);
        cudaFree(c.d_status);
        if (c.h_status) cudaFreeHost(c.h_status);
    }
    cudaFree(s->arena);
    cudaFree(s->d_jd);
    cudaFree(s->d_jm);
    for (Retirer& w : s->retirers) {
        cudaFree(w.d_list);
        sqs_ctx_destroy(w.ctx);
    }
    if (s->ast) cudaStreamDestroy(s->ast);
    if (s->admitted) cudaEventDestroy(s->admitted);
    delete s;
}
}  // namespace

extern "C" int sqs_server_create(sqs_ctx* ctx, size_t hbm_bytes, int max_active, int slice_sweeps,
                                 sqs_server** out) {
    if (int r = enter(ctx)) return r;
    SQS_REQUIRE(out != nullptr, "null output pointer");
    SQS_REQUIRE(max_active >= 1 && max_active <= 4096, "max_active %d out of 1..4096", max_active);
    SQS_REQUIRE(slice_sweeps != 0, "slice_sweeps must be nonzero");
    SQS_REQUIRE(hbm_bytes >= (1u << 20), "hbm budget below 1 MiB");
    sqs_server* s = new sqs_server();
    s->ctx = ctx;
    s->max_active = max_active;
    s->slice = slice_sweeps;
    s->arena_bytes = hbm_bytes & ~(size_t)255;
    cudaError_t e = cudaMalloc(&s->arena, s->arena_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_jd, sizeof(JobDev) * (size_t)max_active);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_jm, sizeof(JobMut) * (size_t)max_active);
    // Each retirement thread (polish, certification) gets its own context on
    // a stream of the highest priority: its blocks are dispatched ahead of
    // pending anneal blocks as SMs free up, so a finished job does not queue
    // behind slices, and batches retire side by side.
    s->retirers.resize(kRetirers);
    for (Retirer& w : s->retirers) {
        if (e != cudaSuccess) break;
        if (int r = sqs_ctx_create(ctx->device, &w.ctx)) {
            free_server(s);
            return r;
        }
        int least = 0, greatest = 0;
        e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
        if (e == cudaSuccess) e = cudaStreamDestroy(w.ctx->stream);
        if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&w.ctx->stream, cudaStreamNonBlocking, greatest);
        if (e == cudaSuccess) e = cudaMalloc(&w.d_list, sizeof(int32_t) * (size_t)max_active);
        // Staging of the certifier, its interval cache and the rescue polish,
        // sized now: growing a buffer later frees the old one, which waits for
        // every slice on the GPU and holds up the caller's thread meanwhile.
        if (e == cudaSuccess && (w.ctx->d_misc.reserve(kRetireStaging) != SQS_OK ||
                                 w.ctx->d_cert.reserve(kRetireCache) != SQS_OK ||
                                 w.ctx->d_polish.reserve(kRetirePolish) != SQS_OK ||
                                 w.ctx->h_cert.reserve(kRetireHost) != SQS_OK))
            e = cudaErrorMemoryAllocation;
    }
    if (e == cudaSuccess) {
        int least = 0, greatest = 0;
        e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
        if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&s->ast, cudaStreamNonBlocking, greatest);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->admitted, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(s->admitted, s->ast);  // waited on before any admission
    }
    s->cohorts.resize(kCohorts);
    for (Cohort& c : s->cohorts) {
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c.st, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaMalloc(&c.d_list, sizeof(int32_t) * (size_t)max_active);
        if (e == cudaSuccess) e = cudaMalloc(&c.d_status, sizeof(int32_t) * (size_t)max_active);
        if (e == cudaSuccess) e = cudaMallocHost(&c.h_status, sizeof(int32_t) * (size_t)max_active);
    }
    if (e != cudaSuccess) {
        set_error("server set-up: %s", cudaGetErrorString(e));
        free_server(s);
        return e == cudaErrorMemoryAllocation ? SQS_ENOMEM : SQS_ECUDA;
    }
    s->free_blocks[0] = s->arena_bytes;
    s->slot_job.assign((size_t)max_active, -1);
    s->flying.assign((size_t)max_active, 0);
    s->retiring.assign((size_t)max_active, 0);
    for (Retirer& w : s->retirers) w.th = std::thread(retire_loop, s, &w);
    *out = s;
    return SQS_OK;
}

extern "C" int sqs_server_destroy(sqs_server* s) {
    if (!s) return SQS_OK;
    cudaSetDevice(s->ctx->device);
    cudaStreamSynchronize(s->ctx->stream);
    free_server(s);
    return SQS_OK;
}

extern "C" int sqs_server_submit(sqs_server* s, const sqs_job* job, int64_t* id) {
    SQS_REQUIRE(s && job && id, "null argument");
    SQS_REQUIRE(job->xya != nullptr || job->n <= 0, "null initial state");
    if (int r = enter(s->ctx)) return r;
    SJob j;
    j.id = s->next_id;
    Shape shape;
    if (int r = resolve_job(s->ctx, *job, 0, j.job, shape)) return r;
    j.xya.assign(job->xya, job->xya + 3 * (size_t)std::max(0, job->n));
    j.job.xya = j.xya.data();
    if (job->xya_rep) {
        j.xya_rep.assign(job->xya_rep, job->xya_rep + 3 * (size_t)std::max(0, job->n) * (size_t)std::max(0, job->replicas));
        j.job.xya_rep = j.xya_rep.data();
    }
    if (int r = prepare_job(j.job, 0, j.jd, j.jm, j.plan, &shape)) return r;
    j.left = job_sweeps(j.job);
    SQS_REQUIRE(job_bytes(j.job) <= s->arena_bytes, "job state (%zu bytes) exceeds the server's HBM budget",
                job_bytes(j.job));
    *id = j.id;
    ++s->next_id;
    const int64_t key = j.id;
    std::lock_guard<std::mutex> lk(s->mu);
    s->jobs.emplace(key, std::move(j));
    SJob& stored = s->jobs[key];
    stored.job.xya = stored.xya.data();  // the vectors moved with the record
    if (stored.job.xya_rep) stored.job.xya_rep = stored.xya_rep.data();
    if (stored.jm.status != kRunning) {   // zero-sweep job: nothing to anneal
        stored.state = kDone;
        fill_result(stored.job, stored.jd, stored.jm, 0.f, stored.res);
    } else {
        s->queue.push_back(key);
    }
    return SQS_OK;
}

namespace {

__global__ void gather_status_kernel(const int32_t* list, int count, const JobMut* jm, int32_t* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) out[i] = jm[list[i]].status;
}

int launch_gather_status(cudaStream_t st, int count, const int32_t* list, const JobMut* jm, int32_t* out) {
    gather_status_kernel<<<(count + 127) / 128, 128, 0, st>>>(list, count, jm, out);
    SQS_CUDA(cudaGetLastError());
    return SQS_OK;
}

// A job's sweeps per slice: its own count under proposal slicing, else the server's.
int job_slice(const sqs_server* s, const SJob& j) { return j.jd.slice > 0 ? j.jd.slice : std::max(1, s->slice); }

// Collect the cohorts whose slice has finished: their jobs become idle again,
// or go to `fin` when their budget is spent (or they failed or were cancelled).
int harvest(sqs_server* s, std::vector<int32_t>& fin, int& got) {
    got = 0;
    for (Cohort& c : s->cohorts) {
        if (!c.busy) continue;
        const cudaError_t e = cudaEventQuery(c.done);
        if (e == cudaErrorNotReady) continue;
        if (e != cudaSuccess) {
            set_error("anneal slice: %s", cudaGetErrorString(e));
            return SQS_ECUDA;
        }
        c.busy = false;
        ++got;
        for (size_t i = 0; i < c.slots.size(); ++i) {
            const int32_t k = c.slots[i];
            s->flying[(size_t)k] = 0;
            if (c.h_status[i] != kRunning || s->jobs[s->slot_job[(size_t)k]].cancel) fin.push_back(k);
        }
        c.slots.clear();
    }
    return SQS_OK;
}

// Start one slice for every idle job: one launch per cluster shape, each on a
// free cohort stream, the jobs with the most work left first (in the launch
// order and in the grid).  Returns the number of launches in `launched`.
int launch_idle(sqs_server* s, const std::vector<int32_t>& fin, int& launched) {
    launched = 0;
    using Key = std::tuple<int, int, int>;
    std::map<Key, std::vector<int32_t>> groups;
    std::map<Key, int64_t> rb;
    std::map<Key, int> nmax;
    std::vector<uint8_t> retiring((size_t)s->max_active, 0);
    for (int32_t k : fin) retiring[(size_t)k] = 1;
    for (int k = 0; k < s->max_active; ++k) {
        if (s->slot_job[(size_t)k] < 0 || s->flying[(size_t)k] || retiring[(size_t)k] || s->retiring[(size_t)k]) continue;
        const SJob& j = s->jobs[s->slot_job[(size_t)k]];
        const Key key = std::make_tuple(j.plan.cs, j.plan.Rl, (int)uses_moves(j.jd.flags));
        groups[key].push_back(k);
        rb[key] = std::max(rb[key], j.plan.rb);
        nmax[key] = std::max(nmax[key], j.job.n);
    }
    auto work = [&](int32_t k) {
        const SJob& j = s->jobs[s->slot_job[(size_t)k]];
        return j.left * (int64_t)j.job.n;
    };
    std::vector<std::pair<int64_t, Key>> order;
    for (auto& g : groups) {
        std::stable_sort(g.second.begin(), g.second.end(), [&](int32_t a, int32_t b) { return work(a) > work(b); });
        order.push_back({work(g.second.front()), g.first});
    }
    std::stable_sort(order.begin(), order.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    for (const auto& o : order) {
        Cohort* c = nullptr;
        for (Cohort& x : s->cohorts)
            if (!x.busy) { c = &x; break; }
        if (!c) break;  // every stream busy: the rest wait for the next step
        const std::vector<int32_t>& list = groups[o.second];
        const int cnt = (int)list.size();
        SQS_CUDA(cudaStreamWaitEvent(c->st, s->admitted, 0));  // the jobs' uploads are done first
        SQS_CUDA(cudaMemcpyAsync(c->d_list, list.data(), sizeof(int32_t) * (size_t)cnt, cudaMemcpyHostToDevice, c->st));
        if (int r = launch_anneal(c->st, cnt, std::get<0>(o.second), std::get<1>(o.second),
                                  anneal_smem(std::get<0>(o.second), std::get<1>(o.second), rb[o.second],
                                              nmax[o.second], std::get<2>(o.second) != 0, cnt),
                                  std::get<2>(o.second) != 0, c->d_list,
                                  s->d_jd, s->d_jm, (float4*)s->arena, (double*)s->arena, std::max(1, s->slice)))
            return r;
        if (int r = launch_gather_status(c->st, cnt, c->d_list, s->d_jm, c->d_status)) return r;
        SQS_CUDA(cudaMemcpyAsync(c->h_status, c->d_status, sizeof(int32_t) * (size_t)cnt, cudaMemcpyDeviceToHost, c->st));
        SQS_CUDA(cudaEventRecord(c->done, c->st));
        c->slots = list;
        c->busy = true;
        for (int32_t k : list) {
            s->flying[(size_t)k] = 1;
            SJob& j = s->jobs[s->slot_job[(size_t)k]];
            j.left = std::max<int64_t>(0, j.left - job_slice(s, j));
        }
        s->ctx->launches += 2;
        ++s->st.slices;
        ++launched;
    }
    return SQS_OK;
}

// Polish, rescue and certify the finished jobs and free their slots and
// arena space.  Runs on the retirement thread, on the retirement context's
// stream, while the caller's thread keeps the cohorts going.  The lock is
// taken only to look the jobs up and to publish the results; in between the
// thread reads job fields that nothing changes while a job is active.
int retire(sqs_server* s, Retirer* me, const std::vector<int32_t>& fin) {
    std::vector<SJob*> jobs;
    std::vector<uint8_t> cancel;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (int32_t k : fin) {
            SJob* j = &s->jobs[s->slot_job[(size_t)k]];
            jobs.push_back(j);
            cancel.push_back(j->cancel ? 1 : 0);
        }
    }
    const int64_t l0 = me->ctx->launches;
    const auto t0 = std::chrono::steady_clock::now();
    size_t psmem = 0;
    for (const SJob* j : jobs) psmem = std::max(psmem, polish_smem_bytes(j->job.n));
    SQS_CUDA(cudaMemcpyAsync(me->d_list, fin.data(), sizeof(int32_t) * fin.size(), cudaMemcpyHostToDevice,
                             me->ctx->stream));
    if (int r = launch_polish(me->ctx->stream, (int)fin.size(), me->d_list, s->d_jd, s->d_jm, (double*)s->arena, psmem))
        return r;
    me->ctx->launches += 1;
    std::vector<std::vector<double>> best(fin.size()), out(fin.size());
    std::vector<JobMut> jm(fin.size());
    for (size_t q = 0; q < fin.size(); ++q) {
        best[q].resize(3 * (size_t)jobs[q]->job.n);
        SQS_CUDA(cudaMemcpyAsync(best[q].data(), (double*)s->arena + jobs[q]->jd.best_off,
                                 sizeof(double) * best[q].size(), cudaMemcpyDeviceToHost, me->ctx->stream));
        SQS_CUDA(cudaMemcpyAsync(&jm[q], s->d_jm + fin[q], sizeof(JobMut), cudaMemcpyDeviceToHost, me->ctx->stream));
    }
    SQS_CUDA(cudaStreamSynchronize(me->ctx->stream));
    const double polish_s = seconds_since(t0);
    {
        std::vector<Rescue> rs;
        for (size_t q = 0; q < fin.size(); ++q)
            if (!cancel[q]) add_rescue(rs, jobs[q]->job, jobs[q]->jd, jm[q], (const float4*)s->arena, best[q].data());
        if (int r = rescue_uncertified(me->ctx, rs)) return r;
    }
    std::vector<sqs_job_result> res(fin.size());
    std::vector<int> ns;
    std::vector<const double*> bptr;
    std::vector<sqs_job_result*> optr;
    std::vector<double*> xptr;
    for (size_t q = 0; q < fin.size(); ++q) {
        fill_result(jobs[q]->job, jobs[q]->jd, jm[q], 0.f, res[q]);
        if (cancel[q]) {
            res[q].status = SQS_ENOTFOUND;
            put(res[q].reason, sizeof res[q].reason, "cancelled");
        }
        out[q].assign(3 * (size_t)jobs[q]->job.n, 0.0);
        if (!cancel[q] && jm[q].status != kErrCells && jm[q].best_L < 1e29) {
            ns.push_back(jobs[q]->job.n);
            bptr.push_back(best[q].data());
            optr.push_back(&res[q]);
            xptr.push_back(out[q].data());
        }
    }
    const auto t1 = std::chrono::steady_clock::now();
    if (int r = certify_states(me->ctx, ns, bptr, optr, xptr)) return r;
    const double certify_s = seconds_since(t1);
    std::lock_guard<std::mutex> lk(s->mu);
    s->st.polish_s += polish_s;
    s->st.certify_s += certify_s;
    for (size_t q = 0; q < fin.size(); ++q) {
        SJob& j = *jobs[q];
        j.res = res[q];
        j.best = std::move(out[q]);
        arena_free(s, j.off, j.bytes);
        j.state = kDone;
        j.slot = -1;
        s->slot_job[(size_t)fin[q]] = -1;
        s->retiring[(size_t)fin[q]] = 0;
    }
    s->st.retired += (int64_t)fin.size();
    s->ctx->launches += me->ctx->launches - l0;
    return SQS_OK;
}

// The retirement thread: retires every batch of finished jobs queued by the
// time it looks, as one batch (jobs that finish while a retirement runs are
// retired together next); an error is kept and reported by the caller's
// next step.
void retire_loop(sqs_server* s, Retirer* me) {
    cudaSetDevice(s->ctx->device);
    for (;;) {
        std::vector<int32_t> fin;
        int64_t batches = 0;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv.wait(lk, [&] { return s->stop || !s->rq.empty(); });
            if (s->rq.empty()) return;  // asked to stop, nothing left
            for (auto& b : s->rq) fin.insert(fin.end(), b.begin(), b.end());
            batches = (int64_t)s->rq.size();
            s->rq.clear();
        }
        const auto t0 = std::chrono::steady_clock::now();
        const int r = retire(s, me, fin);
        std::lock_guard<std::mutex> lk(s->mu);
        if (r && !s->werr) {
            s->werr = r;
            s->werr_msg = sqs_last_error();
        }
        s->st.retire_s += seconds_since(t0);
        s->retire_pending -= batches;
    }
}

}  // namespace

extern "C" int sqs_server_step(sqs_server* s, int* in_flight) {
    SQS_REQUIRE(s != nullptr, "null server");
    if (int r = enter(s->ctx)) return r;
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->werr) {
        set_error("%s", s->werr_msg.c_str());
        return s->werr;
    }
    ++s->st.steps;
    auto t0 = std::chrono::steady_clock::now();
    if (int r = admit(s)) return r;
    s->st.admit_s += seconds_since(t0);
    std::vector<int32_t> fin;
    for (int k = 0; k < s->max_active; ++k)  // cancelled jobs between slices
        if (s->slot_job[(size_t)k] >= 0 && !s->flying[(size_t)k] && !s->retiring[(size_t)k] &&
            s->jobs[s->slot_job[(size_t)k]].cancel)
            fin.push_back(k);
    for (int pass = 0; pass < 2; ++pass) {
        int got = 0, launched = 0;
        const int64_t pend0 = s->retire_pending;
        t0 = std::chrono::steady_clock::now();
        if (int r = harvest(s, fin, got)) return r;
        if (int r = launch_idle(s, fin, launched)) return r;
        s->st.launch_s += seconds_since(t0);
        if (!fin.empty()) {  // hand the finished jobs to the retirement thread
            for (int32_t k : fin) s->retiring[(size_t)k] = 1;
            s->rq.push_back(std::move(fin));
            fin.clear();
            ++s->retire_pending;
            s->cv.notify_one();
            break;
        }
        bool busy = false;
        for (const Cohort& c : s->cohorts) busy = busy || c.busy;
        if (pass == 1 || got || launched || (!busy && !pend0)) break;
        // nothing to do but wait: until a slice or a retirement finishes, at
        // most kWaitSeconds, so that the caller can keep submitting meanwhile
        lk.unlock();
        t0 = std::chrono::steady_clock::now();
        bool ready = false;
        while (!ready && seconds_since(t0) < kWaitSeconds) {
            for (const Cohort& c : s->cohorts) ready = ready || (c.busy && cudaEventQuery(c.done) != cudaErrorNotReady);
            if (!ready) {
                std::this_thread::sleep_for(std::chrono::microseconds(50));
                std::lock_guard<std::mutex> g(s->mu);
                ready = s->retire_pending != pend0;
            }
        }
        lk.lock();
        s->st.wait_s += seconds_since(t0);
    }
    if (in_flight) {
        int active = 0;
        for (int64_t id : s->slot_job) active += id >= 0;
        *in_flight = active + (int)s->queue.size();
    }
    return SQS_OK;
}

extern "C" int sqs_server_poll(sqs_server* s, int64_t id, sqs_job_result* out, double* xya_out) {
    SQS_REQUIRE(s != nullptr && out != nullptr, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) {
        set_error("job %lld unknown (never submitted, or already collected)", (long long)id);
        return SQS_ENOTFOUND;
    }
    if (it->second.state != kDone) return 0;
    *out = it->second.res;
    if (xya_out && out->certified)
        std::memcpy(xya_out, it->second.best.data(), sizeof(double) * it->second.best.size());
    s->jobs.erase(it);
    return 1;
}

extern "C" int sqs_server_cancel(sqs_server* s, int64_t id) {
    SQS_REQUIRE(s != nullptr, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end() || it->second.state == kDone) {
        set_error("job %lld is not queued or running", (long long)id);
        return SQS_ENOTFOUND;
    }
    SJob& j = it->second;
    if (j.state == kQueued) {
        s->queue.erase(std::find(s->queue.begin(), s->queue.end(), id));
        j.state = kDone;
        j.res = sqs_job_result{};
        j.res.status = SQS_ENOTFOUND;
        put(j.res.reason, sizeof j.res.reason, "cancelled");
    } else {
        j.cancel = true;  // retired (uncertified) at the end of the next step
    }
    return SQS_OK;
}

extern "C" int sqs_server_info(sqs_server* s, int* queued, int* active, size_t* hbm_used) {
    SQS_REQUIRE(s != nullptr, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    int a = 0;
    for (int64_t id : s->slot_job) a += id >= 0;
    if (queued) *queued = (int)s->queue.size();
    if (active) *active = a;
    if (hbm_used) *hbm_used = s->used;
    return SQS_OK;
}

extern "C" int sqs_server_get_stats(sqs_server* s, sqs_server_stats* out) {
    SQS_REQUIRE(s && out, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->st;
    return SQS_OK;
}
