// Drop-in for the reference's search programs, on the batched GPU annealer:
//
//   packing seed.txt epochs steps chains random_seed output.json   (packing.cu:768-868)
//   seeded  seed.txt epochs steps chains seed output.json          (seeded.cu:831-983)
//
// Same argument checks (epochs 0..100000, steps 0..4096, chains 0..4096 and
// a multiple of 8; 0 = automatic), same seed-file format ("n L" then n lines
// "x y angle", n <= 1000, 0 < L <= 64), same validated environment variables
// (an out-of-range value prints "invalid NAME" and exits 2), exit code 2 on
// any error, and the same single-line JSON report with the best state in
// "q".  Callers that run these programs (cuda/batch.py, scheduler.run_gpu,
// cpp_loop.case, full_run, demo.main) and read their JSON
// (demo.certified_candidate, seeded.certify_raw, batch.merge,
// autotune.summarize) work unchanged.
//
// Mapping onto sqs_anneal_batch:
//   * every ladder of 8 chains is a ladder of 8 rungs (SQS_JOB_LADDERS), up to
//     8 ladders to a job so that they share one best side, as all of the
//     reference's chains share its bestL; the jobs run side by side in one
//     batched call, and the report takes the smallest certified side;
//   * every rung anneals in its own container below the best,
//     best - shrink * {0.02 .. 20}[rung], restarts ladder heads from a new
//     best and exchanges only in epochs without one (SQS_JOB_TARGETS);
//   * a reference step is one proposal per chain: a job runs epochs * steps
//     proposals per replica and checkpoints (quench, certificate, kick,
//     exchange) after every epoch of `steps` proposals;
//   * the absolute shrink step becomes a relative one (shrink / L);
//   * chains = 0 (or *_AUTOTUNE=1 with chains >= 64) takes one ladder per SM,
//     capped at *_MAX_CHAINS, as the reference sizes chains to a wave;
//     *_AUTOTUNE=1 also lets the launch autotuner pick each job's shape;
//   * temperatures: packing uses PACK_TMIN..PACK_TMAX; seeded uses the
//     reference's fixed 1e-11..SEED_TMAX ladder;
//   * SEED_POLISH is the job's polish budget (packing polishes 200 steps);
//   * the move set is the reference's: step adaptation with the cooling
//     cycle and kicks of overlapped replicas always, collective moves
//     always for packing and under SEED_COLLECTIVE for seeded;
//   * chains start from the structured portfolio (sqs_portfolio, the
//     reference's build_portfolio and structured_init), always for packing
//     and under SEED_STRUCTURED for seeded;
//   * the angle proposal width is 2.5 x the move width (PACK_ROTATION is
//     validated and reported but, as in the reference, not used);
//   * four variables of this build's own, validated like the others:
//     *_TARGETS (0 or 1) selects the target-side ladders above (0: one job per
//     ladder, checkpoints every max(1, round(steps / n)) sweeps, the side
//     shrunk after each certificate by the ladder's place among the
//     reference's 8 offsets), *_QUENCH_ALL (0 or 1) quenches every replica at
//     each checkpoint, *_CERT_ALL (0 or 1) dilation-certifies every replica at
//     each checkpoint whatever its overlap, and *_QUENCH_STEPS (-1..2032) sets
//     the quench iterations per checkpoint with no exit on slow progress (0
//     keeps the library's, -1 takes the polish iterations of the epochs one
//     checkpoint spans); they default to 1, 1, 1, -1.
// "target_L" is the FP64 dilation-certified side of the best state and "q"
// that state (the packing the interval certifier accepted); when no ladder
// finds a certified state the seed is reported with its side, as the
// reference does.  "seconds" times the search call after an untimed call of
// one proposal a replica has loaded the kernels and allocated the buffers,
// as the reference's clock starts after its own set-up.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

#include "sqs.h"

#if defined(SQS_FLAVOR_SEEDED)
static const char* kName = "seeded";
static const char* kPrefix = "SEED_";
#else
static const char* kName = "packing";
static const char* kPrefix = "PACK_";
#endif

// packing parses its variables as float (packing.cu:153-156), seeded as
// double (seeded.cu:819-829); both reject trailing text and out-of-range
// values with "invalid NAME" and exit code 2.
static double env(const char* suffix, double def, double lo, double hi) {
    const std::string name = std::string(kPrefix) + suffix;
    const char* s = std::getenv(name.c_str());
    if (!s) return def;
    char* end = nullptr;
#if defined(SQS_FLAVOR_SEEDED)
    const double v = std::strtod(s, &end);
#else
    const float vf = std::strtof(s, &end);
    const double v = vf;
    lo = (float)lo;
    hi = (float)hi;
#endif
    if (*end || !std::isfinite(v) || v < lo || v > hi) {
        std::cerr << "invalid " << name << "\n";
        std::exit(2);
    }
    return v;
}

// The reference shrinks the chains of a ladder toward 8 different targets,
// L - shrink * {0.02, 0.1, 0.4, 1, 2.5, 5, 10, 20} (seeded.cu:478-481,
// 929-933); here ladder k's job shrinks by the k % 8-th of those steps.
static const double kShrinkMults[8] = {0.02, 0.1, 0.4, 1.0, 2.5, 5.0, 10.0, 20.0};

static int fail(const char* what) {
    std::cerr << kName << ": " << what << ": " << sqs_last_error() << "\n";
    return 2;
}

int main(int argc, char** argv) {
    if (argc != 7) {
        std::cerr << kName << " seed.txt epochs steps chains " << (std::strcmp(kName, "packing") ? "seed" : "random_seed")
                  << " output.json\n";
        return 2;
    }
    int epochs = std::atoi(argv[2]), steps = std::atoi(argv[3]), chains = std::atoi(argv[4]), n = 0;
    if (epochs < 0 || epochs > 100000 || steps < 0 || steps > 4096 || chains < 0 || chains > 4096 ||
        (chains > 0 && chains % 8))
        return 2;
    double L = 0;
    std::ifstream in(argv[1]);
    in >> n >> L;
    if (!in || n < 1 || n > 1000 || !std::isfinite(L) || L <= 0 || L > 64) return 2;
    std::vector<double> seed(3 * (size_t)n);
    for (int i = 0; i < n; ++i) {
        in >> seed[3 * i] >> seed[3 * i + 1] >> seed[3 * i + 2];
        if (!in || !std::isfinite(seed[3 * i]) || !std::isfinite(seed[3 * i + 1]) || !std::isfinite(seed[3 * i + 2]))
            return 2;
    }
#if defined(SQS_FLAVOR_SEEDED)
    const double shrink = env("SHRINK", .001, 1e-7, .1);
    const double tmax = env("TMAX", .0001, 1e-11, .1);
    const double tmin = std::min(1e-11, tmax);
    const double mv = env("MOVE", .02, 1e-6, .3);
    const int collective = (int)env("COLLECTIVE", 1, 0, 1);
    const int polish = (int)env("POLISH", 200, 0, 4096);
    const int structured = (int)env("STRUCTURED", 1, 0, 1);
    const int autotune = (int)env("AUTOTUNE", 1, 0, 1);
    const int max_chains = (int)env("MAX_CHAINS", 768, 8, 4096);
#else
    const double tmin = env("TMIN", 1e-11, 1e-12, 1.0);
    const double tmax = env("TMAX", 1e-4, 1e-12, 1.0);
    const double mv = env("MOVE", .02, .000001, .3);
    (void)env("ROTATION", .12, .000001, 1.57);
    if (tmax < tmin) return 2;
    const double shrink = env("SHRINK", .001, .000001, .1);
    const int autotune = (int)env("AUTOTUNE", 1, 0, 1);
    const int max_chains = (int)env("MAX_CHAINS", 768, 8, 4096);
    const int polish = 200;
    const int collective = 1;  // packing always mixes collective moves in (packing.cu:525)
    const int structured = 1;  // and always starts from the portfolio (packing.cu:806, 821)
#endif
    // options of this build, not the reference's: SQS_JOB_CERT_ALL,
    // SQS_JOB_QUENCH_ALL and SQS_JOB_QUENCH_STEPS on every ladder, all three
    // on by default: the counterparts of the per-epoch uninterrupted polish
    // and certificate of every chain (seeded.cu:621-720, packing.cu:630-689).
    // Quench iterations per checkpoint: 0 = the library's
    // default, -1 = the polish iterations of the epochs one checkpoint spans.
    const int targets = (int)env("TARGETS", 1, 0, 1);
    const int cert_all = (int)env("CERT_ALL", 1, 0, 1);
    const int quench_all = (int)env("QUENCH_ALL", 1, 0, 1);
    const int quench_steps = (int)env("QUENCH_STEPS", -1, -1, 2032);
    const unsigned long long rng_seed = std::strtoull(argv[5], nullptr, 10);

    sqs_ctx* ctx = nullptr;
    if (sqs_ctx_create(0, &ctx) != SQS_OK) return fail("device");
    char dev[256] = {0};
    int sms = 0;
    if (sqs_ctx_device_info(ctx, dev, (int)sizeof dev, &sms) != SQS_OK) return fail("device info");
    const int wave_chains = std::max(8, (sms * 8 / 8) * 8);
    if (chains == 0 || (autotune && chains >= 64)) {
        const int target = chains == 0 ? wave_chains : std::max(chains, std::min(wave_chains, max_chains));
        chains = ((std::min(target, max_chains) + 7) / 8) * 8;
    }
    if (epochs == 0) epochs = n <= 64 ? 50 : (n <= 256 ? 40 : 30);
    if (steps == 0) steps = n <= 64 ? 64 : (n <= 256 ? 48 : 32);
#if !defined(SQS_FLAVOR_SEEDED)
    epochs = epochs > 120 ? std::min(epochs, 80) : epochs;  // packing.cu:805
#endif
    const long long proposals_per_chain = (long long)epochs * steps;
    const int sweeps = (int)std::max<long long>(1, (proposals_per_chain + n - 1) / n);
    const int per_epoch = std::max(1, (int)std::lround((double)steps / (double)n));
    const int ladders = chains / 8;
    int quench_k = 0;  // SQS_JOB_QUENCH_STEPS(k): 16 k iterations
    if (quench_steps > 0) {
        quench_k = (quench_steps + 15) / 16;
    } else if (quench_steps < 0 && polish > 0) {
        // the polish iterations of the epochs one checkpoint spans
        const double iters = targets ? (double)polish : (double)polish * per_epoch * n / steps;
        quench_k = (int)std::min(127.0, std::ceil(iters / 16.0));
    }

    // every chain's start: the structured portfolio (the seed on every chain
    // when SEED_STRUCTURED=0); ladder k's 8 chains are job k's replicas
    std::vector<double> starts(3 * (size_t)n * (size_t)chains);
    if (sqs_portfolio(n, L, seed.data(), chains, structured, rng_seed, 1, starts.data()) != SQS_OK)
        return fail("portfolio");
    // Jobs of `per_job` ladders each (one ladder per job without targets); a
    // job whose ladders do not fit one cluster is retried with half as many.
    std::vector<sqs_job> jobs;
    std::vector<std::vector<double>> outs;
    std::vector<double*> ptrs;
    std::vector<sqs_job_result> res;
    double seconds = 0.0;
    for (int per_job = targets ? std::min(8, ladders) : 1;; per_job = std::max(1, per_job / 2)) {
        const int njobs = (ladders + per_job - 1) / per_job;
        jobs.assign((size_t)njobs, sqs_job{});
        outs.assign((size_t)njobs, std::vector<double>(3 * (size_t)n));
        ptrs.assign((size_t)njobs, nullptr);
        res.assign((size_t)njobs, sqs_job_result{});
        for (int k = 0; k < njobs; ++k) {
            const int lad = std::min(per_job, ladders - k * per_job);  // ladders of this job
            sqs_job& j = jobs[(size_t)k];
            std::memset(&j, 0, sizeof j);
            j.n = n;
            j.replicas = 8 * lad;
            j.polish_iters = polish;
            j.flags = (autotune ? SQS_JOB_AUTOTUNE : 0) | SQS_JOB_ADAPT | SQS_JOB_KICK |
                      (collective ? SQS_JOB_COLLECTIVE : 0) | (cert_all ? SQS_JOB_CERT_ALL : 0) |
                      (quench_all ? SQS_JOB_QUENCH_ALL : 0) | SQS_JOB_QUENCH_STEPS(quench_k);
            if (targets) {
                // epochs * steps proposals, a checkpoint after every epoch
                j.sweeps = (int)std::max<long long>(-2000000000LL, -std::max(1LL, proposals_per_chain));
                j.exchange_every = -std::max(1, steps);
                j.flags |= SQS_JOB_TARGETS | SQS_JOB_LADDERS(lad);
                // without the tuner, the widest cluster (up to 16 CTAs): fewer
                // replicas per CTA leave each replica more warps for its
                // checkpoint quench, as the reference polishes its chains on
                // separate blocks
                if (!autotune) j.flags |= SQS_JOB_CLUSTER(std::min(16, 8 * lad));
                j.shrink = std::min(0.1 / 20.0, shrink / L);
            } else {
                j.sweeps = sweeps;
                j.exchange_every = per_epoch;
                j.shrink = std::min(0.1, shrink * kShrinkMults[k % 8] / L);
            }
            j.L0 = L;
            j.tmin = tmin;
            j.tmax = tmax;
            j.sigma_xy = mv;
            j.sigma_a = std::min(1.0, 0.7 * mv);  // theta = 0.7 scale (seeded.cu:510, packing.cu:531)
            j.seed = rng_seed + 0x9E3779B97F4A7C15ull * (unsigned long long)k;
            j.xya = seed.data();
            j.xya_rep = starts.data() + 3 * (size_t)n * 8 * (size_t)k * (size_t)per_job;
            ptrs[(size_t)k] = outs[(size_t)k].data();
        }
        // Untimed warm-up of one proposal a replica: the first call loads the
        // kernels and allocates the device buffers, which the reference does
        // before it starts its clock (its allocations, copies and first
        // launches precede `start`, seeded.cu:887-906).
        std::vector<sqs_job> warm = jobs;
        for (sqs_job& w : warm) {
            w.sweeps = targets ? -1 : 1;
            w.exchange_every = targets ? -1 : 1;
        }
        (void)sqs_anneal_batch(ctx, warm.data(), njobs, 0, ptrs.data(), res.data());
        const auto t0 = std::chrono::steady_clock::now();
        const int rc = sqs_anneal_batch(ctx, jobs.data(), njobs, 0, ptrs.data(), res.data());
        seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (rc == SQS_OK) break;
        if (rc != SQS_EINVAL || per_job == 1 || !std::strstr(sqs_last_error(), "does not fit")) return fail("anneal");
    }
    const int njobs = (int)jobs.size();

    double bestL = L;
    const double* best = seed.data();
    long long proposals = 0, accepted = 0, xatt = 0, xacc = 0;
    int shrinks = 0, feasible = 0;
    for (int k = 0; k < njobs; ++k) {
        const sqs_job_result& r = res[(size_t)k];
        proposals += r.proposals;
        accepted += r.accepted;
        xatt += r.exchange_attempts;
        xacc += r.exchange_accepts;
        shrinks += r.shrinks;
        feasible += r.improvements;
        if (r.certified && r.L_polished < bestL) {
            bestL = r.L_polished;
            best = outs[(size_t)k].data();
        }
    }
    sqs_ctx_destroy(ctx);

    std::ofstream out(argv[6]);
    if (!out) return 2;
    out << std::setprecision(17);
#if defined(SQS_FLAVOR_SEEDED)
    out << "{\"n\":" << n << ",\"target_L\":" << bestL << ",\"seconds\":" << seconds << ",\"shrinks\":" << shrinks
        << ",\"epochs\":" << epochs << ",\"steps\":" << steps << ",\"chains\":" << chains << ",\"device\":\"" << dev
        << "\"" << ",\"sm_count\":" << sms << ",\"blocks_per_sm\":" << 1 << ",\"wave_chains\":" << wave_chains
        << ",\"collective\":" << collective << ",\"polish\":" << polish << ",\"structured\":" << structured
        << ",\"proposals\":" << proposals << ",\"accepted\":" << accepted << ",\"exchange_attempts\":" << xatt
        << ",\"exchange_accepts\":" << xacc << ",\"q\":[";
#else
    out << "{\"n\":" << n << ",\"target_L\":" << bestL << ",\"seconds\":" << seconds
        << ",\"chain_steps\":" << (long long)chains * epochs * steps << ",\"proposals\":" << proposals
        << ",\"feasible_checkpoints\":" << std::max(1, feasible) << ",\"shrinks\":" << shrinks
        << ",\"chains\":" << chains << ",\"sm_count\":" << sms << ",\"blocks_per_sm\":" << 1
        << ",\"wave_chains\":" << wave_chains << ",\"device\":\"" << dev << "\",\"q\":[";
#endif
    for (int i = 0; i < n; ++i) {
        if (i) out << ",";
        out << "[" << best[3 * i] << "," << best[3 * i + 1] << "," << best[3 * i + 2] << "]";
    }
    out << "]}\n";
    return out ? 0 : 2;
}
