// Host runtime of the annealer: job validation, cluster sizing, device state
// resident in HBM across slices, the slice loop, the FP64 polish launch and
// the certification of every job's best packing on the GPU certifier.
//
// Reference host loops it replaces: seeded.cu:831-983 / packing.cu:768-868
// (argument checks, occupancy-based chain count, per-epoch launches with a
// device-to-host sync and host-side rescaling after every improvement), and
// the Python dilation ladder that turns a raw state into a certified packing
// (polish.certify_q, cuda/polish.py:52-65; demo.certified_candidate,
// cuda/demo.py:25-40).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "anneal_host.h"

namespace sqs {
namespace ann {

constexpr size_t kSmemLimit = 232448 - 4096;  // dynamic shared memory per CTA (static part reserved)

// Smallest cluster (CTAs per job) whose per-CTA replica share fits.
static bool plan_job(int n, int R, double L0, Plan& p) {
    p.Gmax = std::max(1, (int)(L0 / (double)kCellSide));
    p.rb = replica_smem_bytes(n, p.Gmax);
    for (int cs = 1; cs <= 16; ++cs) {
        if (R % cs) continue;
        const int Rl = R / cs;
        if (Rl > kMaxRl) continue;
        if ((int64_t)Rl * p.rb > (int64_t)kSmemLimit) continue;
        p.cs = cs;
        p.Rl = Rl;
        return true;
    }
    return false;
}

static double wrap_quarter(double a) {
    const double q = 1.57079632679489661923;
    a = std::fmod(a, q);
    if (a < 0.0) a += q;
    return a;
}

}  // namespace ann
}  // namespace sqs

extern "C" int sqs_certify_batch(sqs_ctx* ctx, int count, const int32_t* n_of, const int64_t* row_start,
                                 const int32_t* square_id, const char* text, const int64_t* lit_off, int flags,
                                 sqs_verdict* out);

using namespace sqs;
using namespace sqs::ann;

namespace sqs {
namespace ann {
void put(char* dst, size_t cap, const std::string& s) {
    size_t k = std::min(cap - 1, s.size());
    std::memcpy(dst, s.data(), k);
    dst[k] = 0;
}

int prepare_job(const sqs_job& J, int j, JobDev& d, JobMut& m, Plan& p) {
    SQS_REQUIRE(J.n >= 1 && J.n <= kMaxN, "job %d: n=%d out of 1..%d", j, J.n, kMaxN);
    SQS_REQUIRE(J.replicas >= 1 && J.replicas <= kMaxR, "job %d: replicas=%d out of 1..%d", j, J.replicas, kMaxR);
    SQS_REQUIRE(J.sweeps >= 0 && J.sweeps <= 100000000, "job %d: sweeps=%d out of range", j, J.sweeps);
    SQS_REQUIRE(J.exchange_every >= 1, "job %d: exchange_every must be >= 1", j);
    SQS_REQUIRE(std::isfinite(J.L0) && J.L0 > 0 && J.L0 <= 64, "job %d: L0 must be in (0, 64]", j);
    SQS_REQUIRE(J.tmin > 0 && J.tmax >= J.tmin && std::isfinite(J.tmax), "job %d: need 0 < tmin <= tmax", j);
    SQS_REQUIRE(J.sigma_xy > 0 && J.sigma_xy <= 0.3 && J.sigma_a > 0 && J.sigma_a <= 1.0,
                "job %d: sigma out of range", j);
    SQS_REQUIRE(J.shrink >= 0 && J.shrink <= 0.1, "job %d: shrink out of [0, 0.1]", j);
    SQS_REQUIRE(J.polish_iters >= 0 && J.polish_iters <= 100000, "job %d: polish_iters out of range", j);
    SQS_REQUIRE(J.xya != nullptr, "job %d: null initial state", j);
    for (int i = 0; i < 3 * J.n; ++i) SQS_REQUIRE(std::isfinite(J.xya[i]), "job %d: non-finite initial coordinate", j);
    SQS_REQUIRE(plan_job(J.n, J.replicas, J.L0, p), "job %d: n=%d with %d replicas does not fit a cluster of <= 16 CTAs",
                j, J.n, J.replicas);
    std::memset(&d, 0, sizeof d);
    d.n = J.n;
    d.R = J.replicas;
    d.cs = p.cs;
    d.Rl = p.Rl;
    d.sweeps_total = J.sweeps;
    d.exchange_every = J.exchange_every;
    d.Gmax = p.Gmax;
    d.polish_iters = J.polish_iters;
    d.sigma_xy = (float)J.sigma_xy;
    d.sigma_a = (float)J.sigma_a;
    d.tmin = (float)J.tmin;
    d.tmax = (float)J.tmax;
    d.shrink = (float)J.shrink;
    d.L0 = (float)J.L0;
    d.seed = J.seed;
    d.quench_iters = 64;
    std::memset(&m, 0, sizeof m);
    m.L = (float)J.L0;
    m.best_L = 1e30;
    m.status = J.sweeps == 0 ? kFinished : kRunning;
    for (int r = 0; r < J.replicas; ++r) m.perm[r] = r;
    return SQS_OK;
}

int64_t job_pos_elems(const sqs_job& J) { return (int64_t)J.replicas * J.n + 2 * (int64_t)J.n; }

void init_replicas(const sqs_job& J, float4* dst) {
    for (int r = 0; r < J.replicas; ++r)
        for (int i = 0; i < J.n; ++i)
            dst[(int64_t)r * J.n + i] =
                make_float4((float)J.xya[3 * i], (float)J.xya[3 * i + 1], (float)wrap_quarter(J.xya[3 * i + 2]), 0.f);
}

void fill_result(const sqs_job& J, const JobMut& m, float dev_ms, sqs_job_result& o) {
    o.status = m.status == kFinished ? 0 : (m.status < 0 ? m.status : SQS_ETIMEOUT);
    o.shrinks = m.shrinks;
    o.improvements = m.improvements;
    o.sweeps_done = m.sweep;
    o.replicas = J.replicas;
    o.L_cert = m.best_L;
    o.L_polished = m.best_L;
    o.proposals = (int64_t)m.proposals;
    o.accepted = (int64_t)m.accepted;
    o.exchange_attempts = (int64_t)m.xatt;
    o.exchange_accepts = (int64_t)m.xacc;
    o.device_ms = dev_ms;
    o.score = std::ceil(std::sqrt((double)J.n)) / std::sqrt((double)J.n) - 1.0;
    if (m.status == kErrCells) put(o.reason, sizeof o.reason, "cell capacity exceeded (input too dense)");
    else if (m.best_L >= 1e29) put(o.reason, sizeof o.reason, "no feasible state found");
}

// Certify best states through the dilation ladder of polish.certify_q
// (cuda/polish.py:52-65): the first centre dilation in 1+1e-10 .. 1+1e-6
// under which the GPU certifier accepts the packing.  `best[k]` is job k's
// n x 3 FP64 state; results go to out[k] and, when certified, xya_out[k].
int certify_states(sqs_ctx* ctx, const std::vector<int>& ns, const std::vector<const double*>& best,
                   const std::vector<sqs_job_result*>& out, const std::vector<double*>& xya_out) {
    static const double ladder[5] = {1 + 1e-10, 1 + 1e-9, 1 + 1e-8, 1 + 1e-7, 1 + 1e-6};
    std::vector<int> pending;
    for (size_t k = 0; k < ns.size(); ++k) pending.push_back((int)k);
    for (int step = 0; step < 5 && !pending.empty(); ++step) {
        std::vector<int32_t> n_of;
        std::vector<int64_t> row_start{0}, lit_off{0};
        std::string text;
        char buf[64];
        for (int k : pending) {
            const int n = ns[(size_t)k];
            n_of.push_back(n);
            const double* b = best[(size_t)k];
            for (int i = 0; i < n; ++i) {
                const double v[3] = {b[3 * i] * ladder[step], b[3 * i + 1] * ladder[step], b[3 * i + 2]};
                for (double x : v) {
                    std::snprintf(buf, sizeof buf, "%.17g", x);
                    text += buf;
                    lit_off.push_back((int64_t)text.size());
                }
            }
            row_start.push_back(row_start.back() + n);
        }
        std::vector<sqs_verdict> ver(pending.size());
        if (int r = sqs_certify_batch(ctx, (int)pending.size(), n_of.data(), row_start.data(), nullptr, text.data(),
                                      lit_off.data(), 0, ver.data()))
            return r;
        std::vector<int> still;
        for (size_t q = 0; q < pending.size(); ++q) {
            const int k = pending[q];
            sqs_job_result& o = *out[(size_t)k];
            if (ver[q].ok) {
                o.certified = 1;
                o.dilation = ladder[step];
                o.score = ver[q].score;
                put(o.L, sizeof o.L, ver[q].L);
                put(o.reason, sizeof o.reason, "ok");
                if (xya_out[(size_t)k]) {
                    const double* b = best[(size_t)k];
                    for (int i = 0; i < ns[(size_t)k]; ++i) {
                        xya_out[(size_t)k][3 * i] = b[3 * i] * ladder[step];
                        xya_out[(size_t)k][3 * i + 1] = b[3 * i + 1] * ladder[step];
                        xya_out[(size_t)k][3 * i + 2] = b[3 * i + 2];
                    }
                }
            } else {
                still.push_back(k);
                put(o.reason, sizeof o.reason, std::string("certifier: ") + ver[q].reason);
            }
        }
        pending.swap(still);
    }
    return SQS_OK;
}
}  // namespace ann
}  // namespace sqs

extern "C" int sqs_anneal_batch(sqs_ctx* ctx, const sqs_job* jobs, int njobs, int slice_sweeps,
                                double* const* xya_out, sqs_job_result* out) {
    if (int r = enter(ctx)) return r;
    SQS_REQUIRE(njobs >= 0 && (njobs == 0 || (jobs && out)), "bad job array");
    SQS_REQUIRE(slice_sweeps >= 0, "slice_sweeps %d < 0", slice_sweeps);
    if (njobs == 0) return SQS_OK;
    std::vector<JobDev> jd((size_t)njobs);
    std::vector<JobMut> jm((size_t)njobs);
    std::vector<Plan> plan((size_t)njobs);
    int64_t pos_total = 0, best_total = 0;
    for (int j = 0; j < njobs; ++j) {
        std::memset(&out[j], 0, sizeof(sqs_job_result));
        if (int r = prepare_job(jobs[j], j, jd[(size_t)j], jm[(size_t)j], plan[(size_t)j])) return r;
        jd[(size_t)j].pos_off = pos_total;
        jd[(size_t)j].best_off = best_total;
        jd[(size_t)j].scr_off = pos_total + (int64_t)jobs[j].replicas * jobs[j].n;
        pos_total += job_pos_elems(jobs[j]);
        best_total += 3 * (int64_t)jobs[j].n;
    }
    // device state: one allocation, resident for the whole call
    size_t tot = 0;
    auto seg = [&](size_t b) { size_t o = tot; tot += (b + 255) & ~(size_t)255; return o; };
    const size_t o_jd = seg(sizeof(JobDev) * njobs), o_jm = seg(sizeof(JobMut) * njobs);
    const size_t o_pos = seg(sizeof(float4) * (size_t)pos_total), o_best = seg(sizeof(double) * (size_t)best_total);
    const size_t o_list = seg(sizeof(int32_t) * njobs);
    if (int r = ctx->d_anneal.reserve(tot)) return r;
    char* D = (char*)ctx->d_anneal.p;
    JobDev* d_jd = (JobDev*)(D + o_jd);
    JobMut* d_jm = (JobMut*)(D + o_jm);
    float4* d_pos = (float4*)(D + o_pos);
    double* d_best = (double*)(D + o_best);
    int32_t* d_list = (int32_t*)(D + o_list);
    {
        std::vector<float4> hpos((size_t)pos_total);
        std::vector<double> hbest((size_t)best_total, 0.0);
        for (int j = 0; j < njobs; ++j) init_replicas(jobs[j], hpos.data() + jd[(size_t)j].pos_off);
        SQS_CUDA(cudaMemcpyAsync(d_jd, jd.data(), sizeof(JobDev) * njobs, cudaMemcpyHostToDevice, ctx->stream));
        SQS_CUDA(cudaMemcpyAsync(d_jm, jm.data(), sizeof(JobMut) * njobs, cudaMemcpyHostToDevice, ctx->stream));
        SQS_CUDA(cudaMemcpyAsync(d_pos, hpos.data(), sizeof(float4) * hpos.size(), cudaMemcpyHostToDevice, ctx->stream));
        SQS_CUDA(cudaMemcpyAsync(d_best, hbest.data(), sizeof(double) * hbest.size(), cudaMemcpyHostToDevice,
                                 ctx->stream));
        SQS_CUDA(cudaStreamSynchronize(ctx->stream));  // host vectors go out of scope
    }
    // launch groups: jobs sharing (cluster size, replicas per CTA); shared memory of the largest
    std::map<std::pair<int, int>, std::vector<int32_t>> groups;
    for (int j = 0; j < njobs; ++j) groups[{plan[(size_t)j].cs, plan[(size_t)j].Rl}].push_back(j);
    std::vector<int32_t> lists;
    std::vector<std::pair<size_t, size_t>> spans;  // (start, count) in lists
    std::vector<size_t> smems;
    std::vector<std::pair<int, int>> keys;
    for (auto& kv : groups) {
        int64_t rb = 0;
        for (int j : kv.second) rb = std::max(rb, plan[(size_t)j].rb);
        spans.push_back({lists.size(), kv.second.size()});
        lists.insert(lists.end(), kv.second.begin(), kv.second.end());
        smems.push_back((size_t)(rb * kv.first.second));
        keys.push_back(kv.first);
    }
    SQS_CUDA(cudaMemcpyAsync(d_list, lists.data(), sizeof(int32_t) * lists.size(), cudaMemcpyHostToDevice,
                             ctx->stream));
    int max_sweeps = 0, max_xe = 1;
    for (int j = 0; j < njobs; ++j) {
        max_sweeps = std::max(max_sweeps, jobs[j].sweeps);
        max_xe = std::max(max_xe, jobs[j].exchange_every);
    }
    // a slice is a whole number of exchange blocks of every job
    int slice = slice_sweeps > 0 ? slice_sweeps : std::max(1, max_sweeps);
    cudaEvent_t e0 = ctx->ev[62], e1 = ctx->ev[63];
    SQS_CUDA(cudaEventRecord(e0, ctx->stream));
    const int rounds = (max_sweeps + slice - 1) / slice;
    for (int k = 0; k < std::max(1, rounds); ++k) {
        for (size_t g = 0; g < keys.size(); ++g) {
            if (int r = launch_anneal(ctx->stream, (int)spans[g].second, keys[g].first, keys[g].second, smems[g],
                                      d_list + spans[g].first, d_jd, d_jm, d_pos, d_best, slice))
                return r;
            ctx->launches += 1;
        }
    }
    // FP64 gradient polish of every job's best state (jobs with polish_iters > 0)
    size_t psmem = 0;
    for (int j = 0; j < njobs; ++j) psmem = std::max(psmem, polish_smem_bytes(jobs[j].n));
    if (int r = launch_polish(ctx->stream, njobs, d_list, d_jd, d_jm, d_best, psmem)) return r;
    ctx->launches += 1;
    SQS_CUDA(cudaEventRecord(e1, ctx->stream));
    std::vector<double> hbest((size_t)best_total);
    SQS_CUDA(cudaMemcpyAsync(jm.data(), d_jm, sizeof(JobMut) * njobs, cudaMemcpyDeviceToHost, ctx->stream));
    SQS_CUDA(cudaMemcpyAsync(hbest.data(), d_best, sizeof(double) * hbest.size(), cudaMemcpyDeviceToHost,
                             ctx->stream));
    SQS_CUDA(cudaStreamSynchronize(ctx->stream));
    float dev_ms = 0.f;
    SQS_CUDA(cudaEventElapsedTime(&dev_ms, e0, e1));

    // certify every best state
    std::vector<int> ns;
    std::vector<const double*> bptr;
    std::vector<sqs_job_result*> optr;
    std::vector<double*> xptr;
    for (int j = 0; j < njobs; ++j) {
        fill_result(jobs[j], jm[(size_t)j], dev_ms, out[j]);
        const JobMut& m = jm[(size_t)j];
        if (m.status == kErrCells || m.best_L >= 1e29) continue;
        ns.push_back(jobs[j].n);
        bptr.push_back(hbest.data() + jd[(size_t)j].best_off);
        optr.push_back(&out[j]);
        xptr.push_back(xya_out ? xya_out[j] : nullptr);
    }
    if (int r = certify_states(ctx, ns, bptr, optr, xptr)) return r;
    return SQS_OK;
}
