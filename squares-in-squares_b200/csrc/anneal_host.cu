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
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "anneal_host.h"

namespace sqs {
namespace ann {

constexpr size_t kSmemLimit = kAnnealSmemLimit;

// Smallest cluster (CTAs per job), from cs_min up, whose per-CTA replica
// share fits, with cells of side at least `cell`.
static bool plan_job(int n, int R, double L0, float cell, int cs_min, Plan& p) {
    p.cell = cell;
    p.Gmax = std::max(1, (int)(L0 / (double)cell));
    p.rb = replica_smem_bytes(n, p.Gmax);
    for (int cs = std::max(1, cs_min); cs <= 16; ++cs) {
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

extern "C" int sqs_polish_batch(sqs_ctx* ctx, int count, const int32_t* n_of, const double* xya, int iters,
                                double* xya_out, sqs_polish_result* out);
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

int prepare_job(const sqs_job& J, int j, JobDev& d, JobMut& m, Plan& p, const Shape* shape) {
    SQS_REQUIRE(J.n >= 1 && J.n <= kMaxN, "job %d: n=%d out of 1..%d", j, J.n, kMaxN);
    SQS_REQUIRE(J.replicas >= 1 && J.replicas <= kMaxR, "job %d: replicas=%d out of 1..%d", j, J.replicas, kMaxR);
    SQS_REQUIRE(J.sweeps >= -2000000000 && J.sweeps <= 100000000, "job %d: sweeps=%d out of range", j, J.sweeps);
    SQS_REQUIRE(J.exchange_every != 0 && J.exchange_every >= -1000000000,
                "job %d: exchange_every must be nonzero (sweeps, or -proposals)", j);
    const int ladders = std::max(1, (J.flags >> 20) & 0xf);
    SQS_REQUIRE(J.replicas % ladders == 0, "job %d: %d replicas do not split into %d ladders", j, J.replicas, ladders);
    SQS_REQUIRE(std::isfinite(J.L0) && J.L0 > 0 && J.L0 <= 64, "job %d: L0 must be in (0, 64]", j);
    SQS_REQUIRE(J.tmin > 0 && J.tmax >= J.tmin && std::isfinite(J.tmax), "job %d: need 0 < tmin <= tmax", j);
    SQS_REQUIRE(J.sigma_xy > 0 && J.sigma_xy <= 0.3 && J.sigma_a > 0 && J.sigma_a <= 1.0,
                "job %d: sigma out of range", j);
    SQS_REQUIRE(J.shrink >= 0 && J.shrink <= 0.1, "job %d: shrink out of [0, 0.1]", j);
    SQS_REQUIRE(J.polish_iters >= 0 && J.polish_iters <= 100000, "job %d: polish_iters out of range", j);
    SQS_REQUIRE(J.xya != nullptr, "job %d: null initial state", j);
    for (int i = 0; i < 3 * J.n; ++i) SQS_REQUIRE(std::isfinite(J.xya[i]), "job %d: non-finite initial coordinate", j);
    if (J.xya_rep)
        for (int64_t i = 0; i < 3 * (int64_t)J.n * J.replicas; ++i)
            SQS_REQUIRE(std::isfinite(J.xya_rep[i]), "job %d: non-finite replica start", j);
    const bool tuned = shape && shape->cs > 0;
    SQS_REQUIRE(plan_job(J.n, J.replicas, J.L0, tuned ? shape->cell : kCellSide, tuned ? shape->cs : 1, p),
                "job %d: n=%d with %d replicas does not fit a cluster of <= 16 CTAs", j, J.n, J.replicas);
    std::memset(&d, 0, sizeof d);
    d.n = J.n;
    d.R = J.replicas;
    d.cs = p.cs;
    d.Rl = p.Rl;
    d.ladders = ladders;
    d.exchange_every = J.exchange_every;
    d.props_total = job_props(J);
    d.xprops = J.exchange_every > 0 ? (int64_t)J.exchange_every * J.n : -(int64_t)J.exchange_every;
    d.Gmax = p.Gmax;
    d.polish_iters = J.polish_iters;
    d.sigma_xy = (float)J.sigma_xy;
    d.sigma_a = (float)J.sigma_a;
    d.tmin = (float)J.tmin;
    d.tmax = (float)J.tmax;
    d.shrink = (float)J.shrink;
    d.L0 = (float)J.L0;
    d.cell = p.cell;
    d.seed = J.seed;
    // the checkpoint quench: 64 iterations ending after three slow steps, or
    // under SQS_JOB_QUENCH_STEPS(k) 16 k iterations with no slow-step exit
    const int qk = (J.flags >> 24) & 0x7f;
    d.quench_iters = qk ? 16 * qk : 64;
    d.quench_stall = qk ? kQuenchNoStall : 3;
    d.flags = J.flags & (kMoveAdapt | kMoveCollective | kMoveKick | kMoveSerial | kMoveQuenchAll | kCertAll | kTargets);
    std::memset(&m, 0, sizeof m);
    m.L = (float)J.L0;
    m.best_L = 1e30;
    m.status = d.props_total == 0 ? kFinished : kRunning;
    for (int r = 0; r < J.replicas; ++r) {
        m.perm[r] = r;
        m.adapt[r] = 1.0f;
        m.win[r] = 0;
    }
    return SQS_OK;
}

// replicas, then the quench scratch of up to one CTA per replica
int64_t job_pos_elems(const sqs_job& J) { return (int64_t)J.replicas * J.n * (1 + kQuenchScr); }

int64_t job_props(const sqs_job& J) { return J.sweeps >= 0 ? (int64_t)J.sweeps * J.n : -(int64_t)J.sweeps; }

int64_t job_sweeps(const sqs_job& J) { return J.n > 0 ? (job_props(J) + J.n - 1) / J.n : 0; }

void init_replicas(const sqs_job& J, float4* dst) {
    for (int r = 0; r < J.replicas; ++r) {
        const double* src = J.xya_rep ? J.xya_rep + 3 * (size_t)r * J.n : J.xya;
        for (int i = 0; i < J.n; ++i)
            dst[(int64_t)r * J.n + i] =
                make_float4((float)src[3 * i], (float)src[3 * i + 1], (float)wrap_quarter(src[3 * i + 2]), 0.f);
    }
}

void fill_result(const sqs_job& J, const JobDev& d, const JobMut& m, float dev_ms, sqs_job_result& o) {
    o.status = m.status == kFinished ? 0 : (m.status < 0 ? m.status : SQS_ETIMEOUT);
    o.cluster_ctas = d.cs;
    o.replicas_per_cta = d.Rl;
    o.exchange_every = d.exchange_every;
    o.overflows = m.overflows;
    o.cell_side = d.cell;
    o.shrinks = m.shrinks;
    o.improvements = m.improvements;
    o.sweeps_done = (int32_t)(m.done / std::max(1, J.n));
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
int launch_groups(sqs_ctx* ctx, const std::vector<Group>& groups, const JobDev* jdev, JobMut* jmut, float4* pos,
                  double* best, int slice) {
    if (groups.size() == 1) {
        const Group& g = groups[0];
        return launch_anneal(ctx->stream, g.njobs, g.cs, g.Rl, g.smem, g.moves, g.list, jdev, jmut, pos, best, slice);
    }
    const int na = (int)std::min<size_t>(sqs_ctx::kAux, groups.size());
    SQS_CUDA(cudaEventRecord(ctx->fork, ctx->stream));
    for (int a = 0; a < na; ++a) SQS_CUDA(cudaStreamWaitEvent(ctx->aux[a], ctx->fork, 0));
    int rc = SQS_OK;
    for (size_t k = 0; k < groups.size() && rc == SQS_OK; ++k) {
        const Group& g = groups[k];
        rc = launch_anneal(ctx->aux[k % sqs_ctx::kAux], g.njobs, g.cs, g.Rl, g.smem, g.moves, g.list, jdev, jmut, pos, best,
                           slice);
    }
    // join every side stream, also after a failed launch, so the main stream
    // (and a capture in progress) never keeps a dangling branch
    for (int a = 0; a < na; ++a) {
        SQS_CUDA(cudaEventRecord(ctx->join[a], ctx->aux[a]));
        SQS_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->join[a], 0));
    }
    return rc;
}

// ------------------------------------------------------------ autotuner
// Candidate launch shapes of a job: every cluster size that divides the
// replica count and fits, for each cell side; each is timed on the job's own
// initial state (copies of the job fill one wave of the GPU in throughput
// mode; the job runs alone in latency mode) and the fastest wins.  Shape and
// cell side leave the trajectory unchanged (see SQS_JOB_AUTOTUNE), so the
// choice only moves time.  The reference's counterpart is an offline launch
// matrix run as separate processes and summarised afterwards
// (cuda/autotune.py:8-41).
namespace {
struct TuneVal {
    int cs;
    float cell;
    int xe;       // tuned exchange interval (0: not tuned)
    double us;    // device microseconds per sweep
};
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int, int>, TuneVal> g_tune;  // (device, n class, R, mode, exchange tuned)
constexpr float kTuneCells[] = {kCellSide, 1.75f, 1.95f, kCellSideMax};
constexpr int kTuneXe[] = {1, 2, 5, 10, 20, 50, 100};
constexpr size_t kTuneBytes = (size_t)1 << 30;  // trial state cap

int n_class(int n) { return (int)std::floor(4.0 * std::log2((double)n)); }
}  // namespace

// Device milliseconds of `copies` copies of J (sweeps, exchange interval and
// plan fixed), the best of `reps` runs, each from the initial state.
static int trial_ms(sqs_ctx* ctx, const sqs_job& J0, const Plan& p, int copies, int sweeps, int xe, int reps,
                    float* ms) {
    sqs_job J = J0;
    J.sweeps = sweeps;
    J.exchange_every = xe;
    J.polish_iters = 0;
    JobDev d;
    JobMut m;
    Plan q;
    Shape sh;
    sh.cs = p.cs;
    sh.cell = p.cell;
    if (int r = prepare_job(J, 0, d, m, q, &sh)) return r;
    const int64_t pe = job_pos_elems(J);
    size_t tot = 0;
    auto seg = [&](size_t b) { size_t o = tot; tot += (b + 255) & ~(size_t)255; return o; };
    const size_t o_jd = seg(sizeof(JobDev) * copies), o_jm = seg(sizeof(JobMut) * copies);
    const size_t o_pos = seg(sizeof(float4) * (size_t)pe * copies);
    const size_t o_best = seg(sizeof(double) * 3 * (size_t)J.n * copies), o_list = seg(sizeof(int32_t) * copies);
    if (int r = ctx->d_tune.reserve(tot)) return r;
    char* D = (char*)ctx->d_tune.p;
    std::vector<JobDev> jd((size_t)copies, d);
    std::vector<JobMut> jm((size_t)copies, m);
    std::vector<int32_t> list((size_t)copies);
    for (int c = 0; c < copies; ++c) {
        jd[(size_t)c].pos_off = (int64_t)c * pe;
        jd[(size_t)c].scr_off = (int64_t)c * pe + (int64_t)J.replicas * J.n;
        jd[(size_t)c].best_off = (int64_t)c * 3 * J.n;
        list[(size_t)c] = c;
    }
    std::vector<float4> pos((size_t)pe);
    init_replicas(J, pos.data());
    SQS_CUDA(cudaMemcpyAsync(D + o_jd, jd.data(), sizeof(JobDev) * copies, cudaMemcpyHostToDevice, ctx->stream));
    SQS_CUDA(cudaMemcpyAsync(D + o_list, list.data(), sizeof(int32_t) * copies, cudaMemcpyHostToDevice, ctx->stream));
    float best = 1e30f;
    for (int rep = 0; rep < reps; ++rep) {
        SQS_CUDA(cudaMemcpyAsync(D + o_jm, jm.data(), sizeof(JobMut) * copies, cudaMemcpyHostToDevice, ctx->stream));
        for (int c = 0; c < copies; ++c)
            SQS_CUDA(cudaMemcpyAsync(D + o_pos + sizeof(float4) * (size_t)pe * c, pos.data(), sizeof(float4) * pos.size(),
                                     cudaMemcpyHostToDevice, ctx->stream));
        SQS_CUDA(cudaEventRecord(ctx->ev[60], ctx->stream));
        if (int r = launch_anneal(ctx->stream, copies, p.cs, p.Rl, anneal_smem(p.cs, p.Rl, p.rb, J.n, uses_moves(d.flags)),
                                  uses_moves(d.flags), (const int32_t*)(D + o_list),
                                  (const JobDev*)(D + o_jd), (JobMut*)(D + o_jm), (float4*)(D + o_pos),
                                  (double*)(D + o_best), sweeps))
            return r;
        ctx->launches += 1;
        SQS_CUDA(cudaEventRecord(ctx->ev[61], ctx->stream));
        SQS_CUDA(cudaStreamSynchronize(ctx->stream));
        float t = 0.f;
        SQS_CUDA(cudaEventElapsedTime(&t, ctx->ev[60], ctx->ev[61]));
        best = std::min(best, t);
    }
    *ms = best;
    return SQS_OK;
}

static int copies_for(const sqs_job& J, const Plan& p, int mode, int* copies) {
    *copies = 1;
    if (mode & SQS_TUNE_LATENCY) return SQS_OK;
    int waves = 1;
    const bool moves = uses_moves(J.flags & 0xfe);  // option bits above SQS_JOB_AUTOTUNE
    if (int r = anneal_max_clusters(p.cs, p.Rl, anneal_smem(p.cs, p.Rl, p.rb, J.n, moves), moves, &waves)) return r;
    const size_t per = sizeof(float4) * (size_t)job_pos_elems(J) + sizeof(double) * 3 * (size_t)J.n + 1024;
    *copies = (int)std::max<int64_t>(1, std::min<int64_t>(waves, (int64_t)(kTuneBytes / per)));
    return SQS_OK;
}

static int autotune(sqs_ctx* ctx, const sqs_job& job, int mode, sqs_tuning& out) {
    std::memset(&out, 0, sizeof out);
    sqs_job J = job;
    const bool tune_xe = J.exchange_every == 0;
    if (tune_xe) J.exchange_every = 10;  // interval used while shapes are compared
    {
        JobDev d;
        JobMut m;
        Plan p;
        if (int r = prepare_job(J, 0, d, m, p)) return r;  // validates the job
    }
    const auto key = std::make_tuple(ctx->device, n_class(J.n), J.replicas, mode & SQS_TUNE_LATENCY, (int)tune_xe);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune.find(key);
        if (it != g_tune.end()) {
            Plan p;
            // a class member with a larger n may need a larger cluster for the same cell side
            if (plan_job(J.n, J.replicas, J.L0, it->second.cell, it->second.cs, p) ||
                plan_job(J.n, J.replicas, J.L0, it->second.cell, 1, p)) {
                out.cluster_ctas = p.cs;
                out.replicas_per_cta = p.Rl;
                out.cell_side = p.cell;
                out.exchange_every = tune_xe ? it->second.xe : job.exchange_every;
                out.us_per_sweep = it->second.us;
                out.trials = 0;
                return SQS_OK;
            }
        }
    }
    // a trial is a whole number of exchange intervals (the job's own
    // checkpoint frequency), about 2,000 proposals per replica
    const int xe = J.exchange_every;  // sweeps, or (negative) proposals, between checkpoints
    const int want = std::max(2, std::min(100, (2000 + J.n - 1) / J.n));
    const int sweeps = xe > 0 ? std::max(xe, (want + xe - 1) / xe * xe) : want;
    struct Cand {
        Plan p;
        float per_copy;  // throughput mode: device time per job in a full wave; latency mode: time alone
    };
    std::vector<Cand> cands;
    Plan def;
    const bool has_def = plan_job(J.n, J.replicas, J.L0, kCellSide, 1, def);
    int trials = 0;
    auto time_plan = [&](const Plan& p, int reps, float* per_copy) -> int {
        int copies = 1;
        if (int r = copies_for(J, p, mode, &copies)) return r;
        float ms = 0.f;
        if (int r = trial_ms(ctx, J, p, copies, sweeps, xe, reps, &ms)) return r;
        trials += reps;
        *per_copy = ms / (float)copies;
        return SQS_OK;
    };
    // screen every shape once ...
    for (float cell : kTuneCells) {
        for (int cs = 1; cs <= 16; ++cs) {
            Plan p;
            if (!plan_job(J.n, J.replicas, J.L0, cell, cs, p) || p.cs != cs) continue;
            Cand c{p, 0.f};
            if (int r = time_plan(p, 1, &c.per_copy)) return r;
            cands.push_back(c);
        }
    }
    SQS_REQUIRE(!cands.empty(), "autotune: no launch shape fits n=%d with %d replicas", J.n, J.replicas);
    std::sort(cands.begin(), cands.end(), [](const Cand& a, const Cand& b) { return a.per_copy < b.per_copy; });
    // ... then time the two fastest and the default again and keep the best
    // of each; a shape replaces the default only when it is 3% faster
    auto same = [](const Plan& a, const Plan& b) { return a.cs == b.cs && a.cell == b.cell; };
    float def_ms = 1e30f;
    for (size_t k = 0; k < cands.size(); ++k) {
        const bool is_def = has_def && same(cands[k].p, def);
        if (k >= 2 && !is_def) continue;
        float t = 0.f;
        if (int r = time_plan(cands[k].p, 2, &t)) return r;
        cands[k].per_copy = std::min(cands[k].per_copy, t);
        if (is_def) def_ms = cands[k].per_copy;
    }
    Plan best = cands[0].p;
    float best_ms = cands[0].per_copy;
    for (size_t k = 1; k < std::min<size_t>(2, cands.size()); ++k)
        if (cands[k].per_copy < best_ms) {
            best_ms = cands[k].per_copy;
            best = cands[k].p;
        }
    if (has_def && def_ms < 1e29f && !same(best, def) && best_ms > 0.97f * def_ms) {
        best = def;
        best_ms = def_ms;
    }
    int xe_best = job.exchange_every;
    if (tune_xe) {
        // checkpoint cost c and sweep cost s from T sweeps with 1 and with T checkpoints
        const int T = std::max(8, sweeps);
        int copies = 1;
        if (int r = copies_for(J, best, mode, &copies)) return r;
        float a = 0.f, b = 0.f;
        if (int r = trial_ms(ctx, J, best, copies, T, T, 2, &a)) return r;
        if (int r = trial_ms(ctx, J, best, copies, T, 1, 2, &b)) return r;
        trials += 4;
        const double c = std::max(0.0, (double)(b - a) / (double)(T - 1));
        const double sw = std::max(1e-9, ((double)a - c) / (double)T);
        xe_best = kTuneXe[sizeof(kTuneXe) / sizeof(kTuneXe[0]) - 1];
        for (int x : kTuneXe) {
            if (c <= 0.05 * (double)x * sw) {
                xe_best = x;
                break;
            }
        }
    }
    const double us = 1e3 * (double)best_ms / (double)sweeps;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune[key] = TuneVal{best.cs, best.cell, tune_xe ? xe_best : 0, us};
    }
    out.cluster_ctas = best.cs;
    out.replicas_per_cta = best.Rl;
    out.cell_side = best.cell;
    out.exchange_every = xe_best;
    out.us_per_sweep = us;
    out.trials = trials;
    return SQS_OK;
}

int resolve_job(sqs_ctx* ctx, const sqs_job& job, int mode, sqs_job& eff, Shape& shape) {
    eff = job;
    shape = Shape{};
    SQS_REQUIRE(job.flags >= 0, "unknown job flags 0x%x", (unsigned)job.flags);
    const int pin_cs = (job.flags >> 8) & 0xff, pin_cell = (job.flags >> 16) & 0xf;
    if (pin_cs || pin_cell) {
        SQS_REQUIRE(!(job.flags & SQS_JOB_AUTOTUNE), "SQS_JOB_AUTOTUNE and a pinned shape exclude each other");
        SQS_REQUIRE(pin_cs <= 16 && pin_cell < (int)(sizeof(kTuneCells) / sizeof(kTuneCells[0])),
                    "pinned shape out of range (cluster %d, cell index %d)", pin_cs, pin_cell);
        shape.cell = kTuneCells[pin_cell];
        Plan p;
        SQS_REQUIRE(job.n >= 1 && job.n <= kMaxN && job.replicas >= 1 && job.replicas <= kMaxR &&
                        std::isfinite(job.L0) && job.L0 > 0 && job.L0 <= 64,
                    "job out of range");
        SQS_REQUIRE(plan_job(job.n, job.replicas, job.L0, shape.cell, std::max(1, pin_cs), p) &&
                        (pin_cs == 0 || p.cs == pin_cs),
                    "pinned cluster of %d CTAs does not fit n=%d with %d replicas", pin_cs, job.n, job.replicas);
        shape.cs = p.cs;
        return SQS_OK;
    }
    if (!(job.flags & SQS_JOB_AUTOTUNE)) return SQS_OK;
    sqs_tuning t;
    if (int r = autotune(ctx, job, mode, t)) return r;
    shape.cs = t.cluster_ctas;
    shape.cell = (float)t.cell_side;
    if (job.exchange_every == 0) eff.exchange_every = t.exchange_every;
    return SQS_OK;
}

void add_rescue(std::vector<Rescue>& out, const sqs_job& J, const JobDev& d, JobMut& m, const float4* d_pos,
                double* best) {
    if (m.status != kFinished || m.best_L < 1e29 || J.polish_iters <= 0 || job_props(J) <= 0) return;
    int cold = 0;
    for (int r = 0; r < J.replicas; ++r)
        if (m.perm[r] == 0) cold = r;
    out.push_back(Rescue{J.n, J.polish_iters, d_pos + d.pos_off + (int64_t)cold * J.n, best, &m});
}

int rescue_uncertified(sqs_ctx* ctx, const std::vector<Rescue>& items) {
    if (items.empty()) return SQS_OK;
    std::vector<std::vector<float4>> raw(items.size());
    for (size_t k = 0; k < items.size(); ++k) {
        raw[k].resize((size_t)items[k].n);
        SQS_CUDA(cudaMemcpyAsync(raw[k].data(), items[k].d_state, sizeof(float4) * raw[k].size(),
                                 cudaMemcpyDeviceToHost, ctx->stream));
    }
    SQS_CUDA(cudaStreamSynchronize(ctx->stream));
    // one polish batch per distinct budget, so a job's result never depends
    // on what it was batched with
    std::map<int, std::vector<size_t>> by_iters;
    for (size_t k = 0; k < items.size(); ++k) by_iters[items[k].iters].push_back(k);
    for (auto& kv : by_iters) {
        std::vector<int32_t> n_of;
        std::vector<double> xya, out;
        for (size_t k : kv.second) {
            n_of.push_back(items[k].n);
            for (const float4& p : raw[k]) {
                xya.push_back(p.x);
                xya.push_back(p.y);
                xya.push_back(p.z);
            }
        }
        out.resize(xya.size());
        std::vector<sqs_polish_result> res(kv.second.size());
        if (int r = sqs_polish_batch(ctx, (int)n_of.size(), n_of.data(), xya.data(), kv.first, out.data(), res.data()))
            return r;
        size_t row = 0;
        for (size_t q = 0; q < kv.second.size(); ++q) {
            const Rescue& it = items[kv.second[q]];
            if (res[q].L_out < 1e29) {
                std::memcpy(it.best, out.data() + 3 * row, sizeof(double) * 3 * (size_t)it.n);
                it.m->best_L = res[q].L_out;
            }
            row += (size_t)it.n;
        }
    }
    return SQS_OK;
}

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

// sqs_anneal_batch, and with `trace` (one record per job, or NULL) each
// replica's final state read back after the anneal (sqs_anneal_batch_trace).
static int anneal_run(sqs_ctx* ctx, const sqs_job* jobs, int njobs, int slice_sweeps, double* const* xya_out,
                      sqs_job_result* out, sqs_replica_trace* trace) {
    if (int r = enter(ctx)) return r;
    SQS_REQUIRE(njobs >= 0 && (njobs == 0 || (jobs && out)), "bad job array");
    SQS_REQUIRE(slice_sweeps >= 0, "slice_sweeps %d < 0", slice_sweeps);
    if (njobs == 0) return SQS_OK;
    std::vector<JobDev> jd((size_t)njobs);
    std::vector<JobMut> jm((size_t)njobs);
    std::vector<Plan> plan((size_t)njobs);
    std::vector<sqs_job> eff((size_t)njobs);
    int64_t pos_total = 0, best_total = 0;
    const int mode = njobs == 1 ? SQS_TUNE_LATENCY : 0;
    for (int j = 0; j < njobs; ++j) {
        std::memset(&out[j], 0, sizeof(sqs_job_result));
        Shape shape;
        if (int r = resolve_job(ctx, jobs[j], mode, eff[(size_t)j], shape)) return r;
        if (int r = prepare_job(eff[(size_t)j], j, jd[(size_t)j], jm[(size_t)j], plan[(size_t)j], &shape)) return r;
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
    // trace: one (job, replica) item and one record per replica
    int64_t ntrace = 0;
    size_t trace_smem = 0;
    if (trace)
        for (int j = 0; j < njobs; ++j) {
            ntrace += jobs[j].replicas;
            trace_smem = std::max(trace_smem, (size_t)plan[(size_t)j].rb);
        }
    const size_t o_titem = seg(sizeof(int2) * (size_t)ntrace), o_trec = seg(sizeof(TraceRec) * (size_t)ntrace);
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
    // launch groups: jobs sharing (cluster size, replicas per CTA, kernel
    // instance); shared memory of the largest
    std::map<std::tuple<int, int, int>, std::vector<int32_t>> groups;
    for (int j = 0; j < njobs; ++j)
        groups[{plan[(size_t)j].cs, plan[(size_t)j].Rl, (int)uses_moves(jd[(size_t)j].flags)}].push_back(j);
    std::vector<int32_t> lists;
    std::vector<std::pair<size_t, size_t>> spans;  // (start, count) in lists
    std::vector<size_t> smems;
    std::vector<std::tuple<int, int, int>> keys;
    for (auto& kv : groups) {
        int64_t rb = 0;
        int nmax = 1;
        for (int j : kv.second) {
            rb = std::max(rb, plan[(size_t)j].rb);
            nmax = std::max(nmax, jobs[j].n);
        }
        spans.push_back({lists.size(), kv.second.size()});
        lists.insert(lists.end(), kv.second.begin(), kv.second.end());
        smems.push_back(anneal_smem(std::get<0>(kv.first), std::get<1>(kv.first), rb, nmax, std::get<2>(kv.first) != 0,
                                    (int)kv.second.size()));
        keys.push_back(kv.first);
    }
    SQS_CUDA(cudaMemcpyAsync(d_list, lists.data(), sizeof(int32_t) * lists.size(), cudaMemcpyHostToDevice,
                             ctx->stream));
    int max_sweeps = 0, max_xe = 1;
    for (int j = 0; j < njobs; ++j) {
        max_sweeps = std::max(max_sweeps, (int)std::min<int64_t>(job_sweeps(jobs[j]), 1 << 30));
        max_xe = std::max(max_xe, jobs[j].exchange_every);
    }
    // a slice is a whole number of exchange blocks of every job
    int slice = slice_sweeps > 0 ? slice_sweeps : std::max(1, max_sweeps);
    if (int r = prime_anneal()) return r;
    cudaEvent_t e0 = ctx->ev[62], e1 = ctx->ev[63];
    SQS_CUDA(cudaEventRecord(e0, ctx->stream));
    const int rounds = std::max(1, (max_sweeps + slice - 1) / slice);
    std::vector<Group> launch;
    for (size_t g = 0; g < keys.size(); ++g)
        launch.push_back(Group{(int)spans[g].second, std::get<0>(keys[g]), std::get<1>(keys[g]), smems[g],
                               d_list + spans[g].first, std::get<2>(keys[g]) != 0});
    auto one_round = [&]() -> int { return launch_groups(ctx, launch, d_jd, d_jm, d_pos, d_best, slice); };
    if (rounds < 3) {
        for (int k = 0; k < rounds; ++k)
            if (int r = one_round()) return r;
    } else {
        // the slice loop as a CUDA graph: one round (a launch per cluster
        // shape, concurrent branches) captured once and replayed; every
        // launch reads its jobs' progress from device memory, so the replays
        // need no host updates
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        SQS_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        const int rc = one_round();
        const cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
        if (rc != SQS_OK) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        SQS_CUDA(ce);
        cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
        if (ie != cudaSuccess) {
            cudaGraphDestroy(graph);
            SQS_CUDA(ie);
        }
        cudaError_t le = cudaSuccess;
        for (int k = 0; k < rounds && le == cudaSuccess; ++k) le = cudaGraphLaunch(exec, ctx->stream);
        cudaGraphExecDestroy(exec);
        cudaGraphDestroy(graph);
        SQS_CUDA(le);
        ctx->graph_replays += rounds;
    }
    ctx->launches += (int64_t)rounds * (int64_t)keys.size();
    // FP64 gradient polish of every job's best state (jobs with polish_iters > 0)
    size_t psmem = 0;
    for (int j = 0; j < njobs; ++j) psmem = std::max(psmem, polish_smem_bytes(jobs[j].n));
    if (int r = launch_polish(ctx->stream, njobs, d_list, d_jd, d_jm, d_best, psmem)) return r;
    ctx->launches += 1;
    SQS_CUDA(cudaEventRecord(e1, ctx->stream));
    std::vector<TraceRec> trec((size_t)ntrace);
    std::vector<float4> tpos;
    if (ntrace > 0) {
        std::vector<int2> items;
        for (int j = 0; j < njobs; ++j)
            for (int r = 0; r < jobs[j].replicas; ++r) items.push_back(make_int2(j, r));
        SQS_CUDA(cudaMemcpyAsync(D + o_titem, items.data(), sizeof(int2) * items.size(), cudaMemcpyHostToDevice,
                                 ctx->stream));
        if (int r = launch_trace(ctx->stream, (int)ntrace, (const int2*)(D + o_titem), d_jd, d_jm, d_pos,
                                 (TraceRec*)(D + o_trec), trace_smem))
            return r;
        ctx->launches += 1;
        SQS_CUDA(cudaMemcpyAsync(trec.data(), D + o_trec, sizeof(TraceRec) * trec.size(), cudaMemcpyDeviceToHost,
                                 ctx->stream));
        tpos.resize((size_t)pos_total);
        SQS_CUDA(cudaMemcpyAsync(tpos.data(), d_pos, sizeof(float4) * tpos.size(), cudaMemcpyDeviceToHost,
                                 ctx->stream));
    }
    std::vector<double> hbest((size_t)best_total);
    SQS_CUDA(cudaMemcpyAsync(jm.data(), d_jm, sizeof(JobMut) * njobs, cudaMemcpyDeviceToHost, ctx->stream));
    SQS_CUDA(cudaMemcpyAsync(hbest.data(), d_best, sizeof(double) * hbest.size(), cudaMemcpyDeviceToHost,
                             ctx->stream));
    SQS_CUDA(cudaStreamSynchronize(ctx->stream));
    float dev_ms = 0.f;
    SQS_CUDA(cudaEventElapsedTime(&dev_ms, e0, e1));
    if (ntrace > 0) {
        size_t k = 0;
        for (int j = 0; j < njobs; ++j) {
            sqs_replica_trace& t = trace[j];
            const JobMut& m = jm[(size_t)j];
            const int n = jobs[j].n;
            t.exchange_rounds = m.xround;
            t.cells_ok = 1;
            for (int r = 0; r < jobs[j].replicas; ++r, ++k) {
                const TraceRec& q = trec[k];
                t.cells_ok &= q.cells_ok;
                if (t.energy) t.energy[r] = (double)m.E[r] * (1.0 / (double)kEScale);
                if (t.energy_full) t.energy_full[r] = (double)q.E_full * (1.0 / (double)kEScale);
                if (t.L_cert) t.L_cert[r] = q.L_cert;
                if (t.dilation) t.dilation[r] = q.lam;
                if (t.side) t.side[r] = q.side;
                if (t.temperature) t.temperature[r] = q.temp;
                if (t.step_scale) t.step_scale[r] = q.step;
                if (t.rung) t.rung[r] = q.rung;
                if (t.xya) {
                    const float4* src = tpos.data() + jd[(size_t)j].pos_off + (int64_t)r * n;
                    for (int i = 0; i < n; ++i) {
                        t.xya[3 * ((size_t)r * n + i)] = src[i].x;
                        t.xya[3 * ((size_t)r * n + i) + 1] = src[i].y;
                        t.xya[3 * ((size_t)r * n + i) + 2] = src[i].z;
                    }
                }
            }
        }
    }

    // jobs that never certified a state: rescue from the coldest replica
    {
        std::vector<Rescue> rs;
        for (int j = 0; j < njobs; ++j)
            add_rescue(rs, eff[(size_t)j], jd[(size_t)j], jm[(size_t)j], d_pos, hbest.data() + jd[(size_t)j].best_off);
        if (int r = rescue_uncertified(ctx, rs)) return r;
    }
    // certify every best state
    std::vector<int> ns;
    std::vector<const double*> bptr;
    std::vector<sqs_job_result*> optr;
    std::vector<double*> xptr;
    for (int j = 0; j < njobs; ++j) {
        fill_result(eff[(size_t)j], jd[(size_t)j], jm[(size_t)j], dev_ms, out[j]);
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

extern "C" int sqs_anneal_batch(sqs_ctx* ctx, const sqs_job* jobs, int njobs, int slice_sweeps,
                                double* const* xya_out, sqs_job_result* out) {
    return anneal_run(ctx, jobs, njobs, slice_sweeps, xya_out, out, nullptr);
}

extern "C" int sqs_anneal_batch_trace(sqs_ctx* ctx, const sqs_job* jobs, int njobs, int slice_sweeps,
                                      double* const* xya_out, sqs_job_result* out, sqs_replica_trace* trace) {
    SQS_REQUIRE(trace != nullptr || njobs == 0, "null trace array");
    return anneal_run(ctx, jobs, njobs, slice_sweeps, xya_out, out, trace);
}

extern "C" int sqs_autotune(sqs_ctx* ctx, const sqs_job* job, int mode, sqs_tuning* out) {
    if (int r = enter(ctx)) return r;
    SQS_REQUIRE(job && out, "null argument");
    SQS_REQUIRE((mode & ~SQS_TUNE_LATENCY) == 0, "unknown tuning mode %d", mode);
    return autotune(ctx, *job, mode, *out);
}

extern "C" int sqs_polish_batch(sqs_ctx* ctx, int count, const int32_t* n_of, const double* xya, int iters,
                                double* xya_out, sqs_polish_result* out) {
    if (int r = enter(ctx)) return r;
    SQS_REQUIRE(count >= 0, "count %d < 0", count);
    if (count == 0) return SQS_OK;
    SQS_REQUIRE(n_of && xya && xya_out && out, "null host pointer");
    SQS_REQUIRE(iters >= 0 && iters <= 1000000, "iters %d out of 0..1000000", iters);
    std::vector<int64_t> row0((size_t)count + 1, 0);
    int nmax = 1;
    for (int k = 0; k < count; ++k) {
        SQS_REQUIRE(n_of[k] >= 1 && n_of[k] <= kMaxN, "packing %d: n=%d out of 1..%d", k, n_of[k], kMaxN);
        row0[(size_t)k + 1] = row0[(size_t)k] + n_of[k];
        nmax = std::max(nmax, n_of[k]);
    }
    const int64_t rows = row0[(size_t)count];
    for (int64_t i = 0; i < 3 * rows; ++i) SQS_REQUIRE(std::isfinite(xya[i]), "non-finite coordinate at %lld", (long long)i);
    size_t tot = 0;
    auto seg = [&](size_t b) { size_t o = tot; tot += (b + 255) & ~(size_t)255; return o; };
    const size_t o_n = seg(sizeof(int32_t) * count), o_r = seg(sizeof(int64_t) * count);
    const size_t o_x = seg(sizeof(double) * 3 * (size_t)rows), o_res = seg(sizeof(double) * 3 * count);
    if (int r = ctx->d_polish.reserve(tot)) return r;
    char* D = (char*)ctx->d_polish.p;
    SQS_CUDA(cudaMemcpyAsync(D + o_n, n_of, sizeof(int32_t) * count, cudaMemcpyHostToDevice, ctx->stream));
    SQS_CUDA(cudaMemcpyAsync(D + o_r, row0.data(), sizeof(int64_t) * count, cudaMemcpyHostToDevice, ctx->stream));
    SQS_CUDA(cudaMemcpyAsync(D + o_x, xya, sizeof(double) * 3 * (size_t)rows, cudaMemcpyHostToDevice, ctx->stream));
    if (int r = launch_polish_states(ctx->stream, count, (const int32_t*)(D + o_n), (const int64_t*)(D + o_r), iters,
                                     (double*)(D + o_x), (double*)(D + o_res), polish_smem_bytes(nmax)))
        return r;
    ctx->launches += 1;
    std::vector<double> res(3 * (size_t)count);
    SQS_CUDA(cudaMemcpyAsync(xya_out, D + o_x, sizeof(double) * 3 * (size_t)rows, cudaMemcpyDeviceToHost, ctx->stream));
    SQS_CUDA(cudaMemcpyAsync(res.data(), D + o_res, sizeof(double) * res.size(), cudaMemcpyDeviceToHost, ctx->stream));
    SQS_CUDA(cudaStreamSynchronize(ctx->stream));
    for (int k = 0; k < count; ++k) {
        out[k].L_in = res[3 * (size_t)k];
        out[k].L_out = res[3 * (size_t)k + 1];
        out[k].iterations = (int32_t)res[3 * (size_t)k + 2];
        out[k].improved = out[k].L_out < out[k].L_in;
    }
    return SQS_OK;
}

extern "C" int sqs_energy_fp64(sqs_ctx* ctx, int count, const int32_t* n_of, const double* xya, const double* side,
                               double* energy, double* grad) {
    if (int r = enter(ctx)) return r;
    SQS_REQUIRE(count >= 0, "count %d < 0", count);
    if (count == 0) return SQS_OK;
    SQS_REQUIRE(n_of && xya && side && energy, "null host pointer");
    std::vector<int64_t> row0((size_t)count + 1, 0);
    int nmax = 1;
    for (int k = 0; k < count; ++k) {
        SQS_REQUIRE(n_of[k] >= 1 && n_of[k] <= kMaxN, "packing %d: n=%d out of 1..%d", k, n_of[k], kMaxN);
        SQS_REQUIRE(std::isfinite(side[k]) && side[k] > 0, "packing %d: side must be finite and positive", k);
        row0[(size_t)k + 1] = row0[(size_t)k] + n_of[k];
        nmax = std::max(nmax, n_of[k]);
    }
    const int64_t rows = row0[(size_t)count];
    for (int64_t i = 0; i < 3 * rows; ++i) SQS_REQUIRE(std::isfinite(xya[i]), "non-finite coordinate at %lld", (long long)i);
    size_t tot = 0;
    auto seg = [&](size_t b) { size_t o = tot; tot += (b + 255) & ~(size_t)255; return o; };
    const size_t o_n = seg(sizeof(int32_t) * count), o_r = seg(sizeof(int64_t) * count);
    const size_t o_s = seg(sizeof(double) * count), o_x = seg(sizeof(double) * 3 * (size_t)rows);
    const size_t o_e = seg(sizeof(double) * count), o_g = seg(grad ? sizeof(double) * 3 * (size_t)rows : 0);
    if (int r = ctx->d_polish.reserve(tot)) return r;
    char* D = (char*)ctx->d_polish.p;
    SQS_CUDA(cudaMemcpyAsync(D + o_n, n_of, sizeof(int32_t) * count, cudaMemcpyHostToDevice, ctx->stream));
    SQS_CUDA(cudaMemcpyAsync(D + o_r, row0.data(), sizeof(int64_t) * count, cudaMemcpyHostToDevice, ctx->stream));
    SQS_CUDA(cudaMemcpyAsync(D + o_s, side, sizeof(double) * count, cudaMemcpyHostToDevice, ctx->stream));
    SQS_CUDA(cudaMemcpyAsync(D + o_x, xya, sizeof(double) * 3 * (size_t)rows, cudaMemcpyHostToDevice, ctx->stream));
    if (int r = launch_energy_states(ctx->stream, count, (const int32_t*)(D + o_n), (const int64_t*)(D + o_r),
                                     (const double*)(D + o_s), (const double*)(D + o_x), (double*)(D + o_e),
                                     grad ? (double*)(D + o_g) : nullptr, energy_smem_bytes(nmax)))
        return r;
    ctx->launches += 1;
    SQS_CUDA(cudaMemcpyAsync(energy, D + o_e, sizeof(double) * count, cudaMemcpyDeviceToHost, ctx->stream));
    if (grad)
        SQS_CUDA(cudaMemcpyAsync(grad, D + o_g, sizeof(double) * 3 * (size_t)rows, cudaMemcpyDeviceToHost, ctx->stream));
    SQS_CUDA(cudaStreamSynchronize(ctx->stream));
    return SQS_OK;
}
