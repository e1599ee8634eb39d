// Serving runtime: a continuous-batching request loop for anneal-and-certify
// jobs on one GPU.
//
//   submit   copies a job into the queue (no device work);
//   step     one round of the loop:
//              admit queued jobs while a job slot is free and the job's state
//              (R*n replica squares + quench scratch + FP64 best) fits the HBM
//              arena (first fit, looking past a job that does not fit yet);
//              one anneal slice for every admitted job in a single launch per
//              cluster shape -- jobs admitted at different times, at different
//              sweep counts, run side by side, their state resident in HBM
//              between slices;
//              the jobs whose budget ran out are polished, certified and
//              retired, and their slot and arena space go to the next;
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
#include <cstring>
#include <deque>
#include <map>
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
    size_t off = 0, bytes = 0;  // arena block
    sqs_job_result res{};
    std::vector<double> best;   // certified packing (n x 3) when done
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
    int32_t* d_list = nullptr;
    std::vector<int64_t> slot_job;         // job id per slot, -1 free
    std::deque<int64_t> queue;
    std::unordered_map<int64_t, SJob> jobs;
    int64_t next_id = 1;
    std::vector<JobMut> h_jm;
    size_t used = 0;
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

size_t job_bytes(const sqs_job& J) {
    const size_t b = sizeof(float4) * (size_t)job_pos_elems(J) + sizeof(double) * 3 * (size_t)J.n;
    return (b + 255) & ~(size_t)255;
}

int admit(sqs_server* s) {
    const size_t window = 16;  // look past jobs that do not fit yet
    size_t looked = 0;
    for (auto it = s->queue.begin(); it != s->queue.end() && looked < window;) {
        ++looked;
        SJob& j = s->jobs[*it];
        int slot = -1;
        for (int k = 0; k < s->max_active; ++k)
            if (s->slot_job[(size_t)k] < 0) { slot = k; break; }
        if (slot < 0) break;
        const size_t bytes = job_bytes(j.job);
        const size_t off = arena_alloc(s, bytes);
        if (off == (size_t)-1) { ++it; continue; }
        j.off = off;
        j.bytes = bytes;
        j.slot = slot;
        j.state = kActive;
        j.jd.pos_off = (int64_t)(off / sizeof(float4));
        j.jd.scr_off = j.jd.pos_off + (int64_t)j.job.replicas * j.job.n;
        j.jd.best_off = (int64_t)((off + sizeof(float4) * (size_t)job_pos_elems(j.job)) / sizeof(double));
        if (s->slice < 0) {  // this job's sweeps per step: about -slice proposals, whole exchange intervals
            const int xe = j.jd.exchange_every;
            const int64_t sw = std::max<int64_t>(1, (-(int64_t)s->slice + j.job.n - 1) / j.job.n);
            j.jd.slice = (int)std::min<int64_t>((sw + xe - 1) / xe * xe, 1 << 30);
        }
        std::vector<float4> init((size_t)job_pos_elems(j.job), make_float4(0.f, 0.f, 0.f, 0.f));
        init_replicas(j.job, init.data());
        SQS_CUDA(cudaMemcpyAsync(s->arena + off, init.data(), sizeof(float4) * init.size(), cudaMemcpyHostToDevice,
                                 s->ctx->stream));
        SQS_CUDA(cudaMemcpyAsync(s->d_jd + slot, &j.jd, sizeof(JobDev), cudaMemcpyHostToDevice, s->ctx->stream));
        SQS_CUDA(cudaMemcpyAsync(s->d_jm + slot, &j.jm, sizeof(JobMut), cudaMemcpyHostToDevice, s->ctx->stream));
        SQS_CUDA(cudaStreamSynchronize(s->ctx->stream));  // `init` is a host temporary
        s->slot_job[(size_t)slot] = j.id;
        it = s->queue.erase(it);
    }
    return SQS_OK;
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
    if (e == cudaSuccess) e = cudaMalloc(&s->d_list, sizeof(int32_t) * (size_t)max_active);
    if (e != cudaSuccess) {
        set_error("server set-up: %s", cudaGetErrorString(e));
        cudaFree(s->arena);
        cudaFree(s->d_jd);
        cudaFree(s->d_jm);
        cudaFree(s->d_list);
        delete s;
        return e == cudaErrorMemoryAllocation ? SQS_ENOMEM : SQS_ECUDA;
    }
    s->free_blocks[0] = s->arena_bytes;
    s->slot_job.assign((size_t)max_active, -1);
    s->h_jm.resize((size_t)max_active);
    *out = s;
    return SQS_OK;
}

extern "C" int sqs_server_destroy(sqs_server* s) {
    if (!s) return SQS_OK;
    cudaSetDevice(s->ctx->device);
    cudaStreamSynchronize(s->ctx->stream);
    cudaFree(s->arena);
    cudaFree(s->d_jd);
    cudaFree(s->d_jm);
    cudaFree(s->d_list);
    delete s;
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
    SQS_REQUIRE(job_bytes(j.job) <= s->arena_bytes, "job state (%zu bytes) exceeds the server's HBM budget",
                job_bytes(j.job));
    *id = j.id;
    ++s->next_id;
    const int64_t key = j.id;
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

extern "C" int sqs_server_step(sqs_server* s, int* in_flight) {
    SQS_REQUIRE(s != nullptr, "null server");
    if (int r = enter(s->ctx)) return r;
    if (int r = admit(s)) return r;
    // one slice for every admitted job, one launch per cluster shape
    std::map<std::tuple<int, int, int>, std::vector<int32_t>> groups;
    std::map<std::tuple<int, int, int>, int64_t> rb;
    for (int k = 0; k < s->max_active; ++k) {
        if (s->slot_job[(size_t)k] < 0) continue;
        const SJob& j = s->jobs[s->slot_job[(size_t)k]];
        const auto key = std::make_tuple(j.plan.cs, j.plan.Rl, (int)(j.jd.flags != 0));
        groups[key].push_back(k);
        rb[key] = std::max(rb[key], j.plan.rb);
    }
    std::vector<int32_t> lists;
    std::vector<std::pair<size_t, size_t>> spans;
    for (auto& g : groups) {
        spans.push_back({lists.size(), g.second.size()});
        lists.insert(lists.end(), g.second.begin(), g.second.end());
    }
    if (!lists.empty()) {
        SQS_CUDA(cudaMemcpyAsync(s->d_list, lists.data(), sizeof(int32_t) * lists.size(), cudaMemcpyHostToDevice,
                                 s->ctx->stream));
        std::vector<Group> launch;
        size_t gi = 0;
        for (auto& g : groups) {
            launch.push_back(Group{(int)spans[gi].second, std::get<0>(g.first), std::get<1>(g.first),
                                   (size_t)(rb[g.first] * std::get<1>(g.first)), s->d_list + spans[gi].first,
                                   std::get<2>(g.first) != 0});
            ++gi;
        }
        if (int r = launch_groups(s->ctx, launch, s->d_jd, s->d_jm, (float4*)s->arena, (double*)s->arena,
                                  std::max(1, s->slice)))
            return r;
        s->ctx->launches += (int64_t)launch.size();
        SQS_CUDA(cudaMemcpyAsync(s->h_jm.data(), s->d_jm, sizeof(JobMut) * (size_t)s->max_active,
                                 cudaMemcpyDeviceToHost, s->ctx->stream));
        SQS_CUDA(cudaStreamSynchronize(s->ctx->stream));
    }
    // retire the jobs whose budget is spent (or that failed, or were cancelled)
    std::vector<int32_t> fin;
    for (int k = 0; k < s->max_active; ++k) {
        if (s->slot_job[(size_t)k] < 0) continue;
        const SJob& j = s->jobs[s->slot_job[(size_t)k]];
        if (s->h_jm[(size_t)k].status != kRunning || j.cancel) fin.push_back(k);
    }
    if (!fin.empty()) {
        size_t psmem = 0;
        for (int k : fin) psmem = std::max(psmem, polish_smem_bytes(s->jobs[s->slot_job[(size_t)k]].job.n));
        SQS_CUDA(cudaMemcpyAsync(s->d_list, fin.data(), sizeof(int32_t) * fin.size(), cudaMemcpyHostToDevice,
                                 s->ctx->stream));
        if (int r = launch_polish(s->ctx->stream, (int)fin.size(), s->d_list, s->d_jd, s->d_jm, (double*)s->arena,
                                  psmem))
            return r;
        s->ctx->launches += 1;
        std::vector<std::vector<double>> best(fin.size());
        for (size_t q = 0; q < fin.size(); ++q) {
            SJob& j = s->jobs[s->slot_job[(size_t)fin[q]]];
            best[q].resize(3 * (size_t)j.job.n);
            SQS_CUDA(cudaMemcpyAsync(best[q].data(), (double*)s->arena + j.jd.best_off, sizeof(double) * best[q].size(),
                                     cudaMemcpyDeviceToHost, s->ctx->stream));
        }
        SQS_CUDA(cudaMemcpyAsync(s->h_jm.data(), s->d_jm, sizeof(JobMut) * (size_t)s->max_active,
                                 cudaMemcpyDeviceToHost, s->ctx->stream));
        SQS_CUDA(cudaStreamSynchronize(s->ctx->stream));
        {
            std::vector<Rescue> rs;
            for (size_t q = 0; q < fin.size(); ++q) {
                SJob& j = s->jobs[s->slot_job[(size_t)fin[q]]];
                if (!j.cancel)
                    add_rescue(rs, j.job, j.jd, s->h_jm[(size_t)fin[q]], (const float4*)s->arena, best[q].data());
            }
            if (int r = rescue_uncertified(s->ctx, rs)) return r;
        }
        std::vector<int> ns;
        std::vector<const double*> bptr;
        std::vector<sqs_job_result*> optr;
        std::vector<double*> xptr;
        for (size_t q = 0; q < fin.size(); ++q) {
            SJob& j = s->jobs[s->slot_job[(size_t)fin[q]]];
            j.res = sqs_job_result{};
            fill_result(j.job, j.jd, s->h_jm[(size_t)fin[q]], 0.f, j.res);
            if (j.cancel) {
                j.res.status = SQS_ENOTFOUND;
                put(j.res.reason, sizeof j.res.reason, "cancelled");
            }
            j.best.assign(3 * (size_t)j.job.n, 0.0);
            const JobMut& m = s->h_jm[(size_t)fin[q]];
            if (!j.cancel && m.status != kErrCells && m.best_L < 1e29) {
                ns.push_back(j.job.n);
                bptr.push_back(best[q].data());
                optr.push_back(&j.res);
                xptr.push_back(j.best.data());
            }
        }
        if (int r = certify_states(s->ctx, ns, bptr, optr, xptr)) return r;
        for (int k : fin) {
            SJob& j = s->jobs[s->slot_job[(size_t)k]];
            arena_free(s, j.off, j.bytes);
            j.state = kDone;
            j.slot = -1;
            s->slot_job[(size_t)k] = -1;
        }
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
    int a = 0;
    for (int64_t id : s->slot_job) a += id >= 0;
    if (queued) *queued = (int)s->queue.size();
    if (active) *active = a;
    if (hbm_used) *hbm_used = s->used;
    return SQS_OK;
}
