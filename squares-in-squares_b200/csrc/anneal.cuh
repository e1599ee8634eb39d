// Device-side job records of the batched parallel-tempering annealer, shared
// by the anneal and polish kernels and the host runtime (anneal_host.cu).
#pragma once
#include <cstdint>

namespace sqs {
namespace ann {

constexpr int kMaxR = 64;            // replicas (temperature rungs) per job
constexpr int kMaxRl = 16;           // replicas (warps) per CTA: 512 threads, 128 registers each
constexpr int kCellK = 12;           // slot capacity of one cell
constexpr float kCellSide = 1.59f;   // >= sqrt(2.000001) + largest centre move (0.12 * sqrt 2)
constexpr float kCellSideMax = 2.2f; // largest cell side the autotuner tries
constexpr float kMaxStep = 0.12f;    // clamp of each proposal coordinate
constexpr int kMaxN = 1000;
// float4 scratch per square of one checkpoint quench (gradient sums,
// previous gradient, direction, saved state, and 8 words a square for the
// line search's pair list)
constexpr int kQuenchScr = 6;
// JobDev.quench_stall of SQS_JOB_QUENCH_STEPS jobs: no exit on slow progress.
constexpr int32_t kQuenchNoStall = 0x7fffffff;

// Per job, read-only while a slice runs.
struct JobDev {
    int32_t n, R, cs, Rl;             // squares, replicas, CTAs per job (cluster size), replicas per CTA
    int32_t ladders, exchange_every;  // ladders of R / ladders rungs each; the job's exchange_every (as given)
    int32_t Gmax, polish_iters;       // cell grid side for the initial container; polish iterations
    float sigma_xy, sigma_a, tmin, tmax;
    float shrink, L0, cell, pad1;     // cell: minimum cell side of the cell lists (>= kCellSide)
    uint64_t seed;
    int64_t pos_off;                  // float4 index of replica 0, square 0
    int64_t best_off;                 // double index of the best state (n x 3)
    int64_t scr_off;                  // float4 index of the job's quench scratch (kQuenchScr n per CTA)
    int64_t props_total;              // proposals per replica in the job's budget
    int64_t xprops;                   // proposals per replica between checkpoints
    int32_t quench_iters, flags;      // gradient steps of a checkpoint quench (at most); kMove* bits
    int32_t slice;                    // sweeps per launch for this job (0: the launch's slice)
    int32_t quench_stall;             // accepted slow steps (< 0.1% gained each) that end a quench
};

// Move-set options of a job (the same bits as SQS_JOB_ADAPT, _COLLECTIVE, _KICK).
// kMoveSerial selects the one-at-a-time kernel instance and changes nothing else;
// kCertAll (SQS_JOB_CERT_ALL) only drops the energy gate of the checkpoint's
// dilation certificate and keeps the kernel instance the other bits select
// kTargets (SQS_JOB_TARGETS) gives every rung its own side below the best and
// also selects the move-set instance, which holds the per-replica sides.
enum : int32_t { kMoveAdapt = 2, kMoveCollective = 4, kMoveKick = 8, kMoveSerial = 16, kMoveQuenchAll = 32,
                 kCertAll = 64, kTargets = 128 };

// Whether a job's flags select the move-set kernel instance.
inline bool uses_moves(int32_t flags) { return (flags & ~kCertAll) != 0; }

// The reference's ladder of target offsets: rung b % 8 of a ladder anneals at
// best - shrink * {0.02, 0.1, 0.4, 1, 2.5, 5, 10, 20}[b % 8] (seeded.cu:478-481).
// A ladder of RL rungs takes entry round(7 pos / (RL - 1)) for its rung pos.
__host__ __device__ inline float target_mult(int pos, int RL) {
    const float m[8] = {0.02f, 0.1f, 0.4f, 1.0f, 2.5f, 5.0f, 10.0f, 20.0f};
    if (RL <= 1) return 1.0f;
    return m[(pos * 7 + (RL - 1) / 2) / (RL - 1)];
}

// Per job, advanced by every slice.
struct JobMut {
    float L;                          // container side (SQS_JOB_TARGETS: the best side the rung sides hang from)
    int32_t xround;                   // exchange rounds completed
    int32_t status;                   // 0 running, 1 finished, < 0 error
    int32_t shrinks, improvements;
    int32_t overflows;                // moves rejected because the target cell was full
    int64_t done;                     // proposals per replica completed
    double best_L;                    // best FP64 dilation-certified side (1e30: none yet)
    uint64_t proposals, accepted, xatt, xacc;
    int32_t perm[kMaxR];              // rung (temperature index) of each replica
    int64_t E[kMaxR];                 // energy of each replica, fixed point (kEScale units)
    float adapt[kMaxR];               // step-size adaptation factor of each replica (kMoveAdapt)
    int32_t win[kMaxR];               // accepted proposals in its current window of 16
};

// One replica's final state as sqs_anneal_batch_trace reports it.
struct TraceRec {
    long long E_full;   // fixed-point energy recomputed from scratch (kEScale units)
    double L_cert;      // FP64 dilation-certified side (1e9: dilation above 1.008)
    double lam;         // that dilation
    float temp;         // temperature of its next proposal (rung temperature x cooling)
    float step;         // its step scale (SQS_JOB_ADAPT; else 1)
    float side;         // container side its energy is measured in
    int32_t rung;       // temperature index
    int32_t cells_ok;   // its cell list fitted
    int32_t pad;
};
// Energies are accumulated as integers in units of 2^-40: every pair and
// wall term is rounded once, so sums are exact and independent of the order
// in which neighbours are visited (cell lists are rebuilt with atomics), and
// the running energy of a replica never drifts from its full recomputation.
constexpr float kEScale = 1099511627776.0f;  // 2^40

enum : int32_t { kRunning = 0, kFinished = 1, kErrCells = -2, kErrInput = -3 };

// Dynamic shared memory a CTA of the annealer may ask for (the static part reserved).
constexpr size_t kAnnealSmemLimit = 232448 - 4096;

// Shared-memory bytes one replica needs: (x, y, cos, sin), angle, cell counts, cell slots.
__host__ __device__ inline int64_t replica_smem_bytes(int n, int Gmax) {
    int64_t b = (int64_t)n * 16 + (int64_t)n * 4;
    b += ((int64_t)Gmax * Gmax + 3) & ~3LL;
    b += (int64_t)Gmax * Gmax * kCellK * 2;
    return (b + 15) & ~15LL;
}

}  // namespace ann
}  // namespace sqs
