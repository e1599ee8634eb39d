/*
 * libsqs -- B200 (sm_100a) engine for packing n unit squares into the
 * smallest square: SAT overlap energy, parallel-tempering annealing, FP64
 * best-state recompute, gradient polish and interval certification.
 *
 * C ABI.  Every call returns 0 on success or a negative SQS_E* code, and then
 * sqs_last_error() (per calling thread) holds a one-line message.  Buffers
 * are owned by the caller.  A context owns one CUDA stream on one device;
 * calls on one context are serialised by the caller (one thread at a time),
 * distinct contexts may be used from distinct threads.
 *
 * The reference drives the same work through process and file protocols
 * rather than an in-process API; each entry point below names the
 * reference interface it replaces.
 */
#ifndef SQS_H
#define SQS_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SQS_OK 0
#define SQS_EINVAL (-1)   /* argument out of range (reference: exit code 2) */
#define SQS_ECUDA (-2)    /* CUDA runtime error                              */
#define SQS_ENOMEM (-3)   /* device or host allocation failed                */
#define SQS_ETIMEOUT (-4) /* an iteration-limited device loop ran out        */
#define SQS_EBUSY (-5)    /* serving queue full / admission refused          */
#define SQS_ENOTFOUND (-6)/* unknown job handle                              */

typedef struct sqs_ctx sqs_ctx;

/* ------------------------------------------------------------- plumbing */
/* Library version string. */
const char* sqs_version(void);
/* Message of the last failed call on this thread ("" if none). */
const char* sqs_last_error(void);
/* Number of visible CUDA devices (0 when none; never fails). */
int sqs_device_count(void);
/* Context on `device` with its own stream.  Replaces the per-process CUDA
 * set-up of packing.cu:788 / seeded.cu:858 (device properties, occupancy). */
int sqs_ctx_create(int device, sqs_ctx** out);
int sqs_ctx_destroy(sqs_ctx* ctx);
/* Device properties the reference prints into its raw JSON (seeded.cu:958-961). */
int sqs_ctx_device_info(sqs_ctx* ctx, char* name, int name_cap, int* sm_count);
/* Device memory for callers that keep batches resident in HBM. */
int sqs_dev_alloc(sqs_ctx* ctx, size_t bytes, void** dptr);
int sqs_dev_free(sqs_ctx* ctx, void* dptr);
/* Stream-ordered copies on the context stream (host side may be pageable). */
int sqs_copy_h2d(sqs_ctx* ctx, void* dst, const void* src, size_t bytes);
int sqs_copy_d2h(sqs_ctx* ctx, void* dst, const void* src, size_t bytes);
int sqs_memset(sqs_ctx* ctx, void* dst, int value, size_t bytes);
/* Page-locked host memory (for timed host<->device transfers). */
int sqs_host_alloc(size_t bytes, void** hptr);
int sqs_host_free(void* hptr);
int sqs_sync(sqs_ctx* ctx);
/* Timing on the context stream: record event `slot` (0..63); elapsed ms
 * between two recorded slots (synchronises on `b`). */
int sqs_event_record(sqs_ctx* ctx, int slot);
int sqs_event_elapsed(sqs_ctx* ctx, int a, int b, float* ms);
/* Overwrite a 256 MiB device buffer (twice the 126 MB L2) so the next
 * launch reads its inputs from HBM. */
int sqs_flush_l2(sqs_ctx* ctx);
/* Device memory now free and in total (cudaMemGetInfo), and the bytes the
 * context's own staging buffers hold on the device and in pinned host memory
 * (they only grow, and are released by sqs_ctx_destroy).  Any pointer may be
 * NULL. */
int sqs_ctx_memory(sqs_ctx* ctx, size_t* device_free, size_t* device_total, size_t* staging_device,
                   size_t* staging_host);
/* Kernel launches this context issued since creation (all of libsqs's own
 * kernels; library copies/memsets are not counted). */
int64_t sqs_launch_count(sqs_ctx* ctx);
/* Replays of captured CUDA graphs (the annealer's slice loop) on ctx. */
int64_t sqs_graph_replay_count(sqs_ctx* ctx);

/* --------------------------------------------------------- SAT energy */
/* FP32 cell-list SAT overlap + wall energy and gradient of `configs`
 * independent configurations of n unit squares (n <= 1024), device pointers:
 *   xya    [configs][n][3] float  centre x, centre y, angle (radians)
 *   side   [configs]       float  container side L
 *   energy [configs]       float  walls + sum_{i<j} pair
 *   grad   [configs][n][3] float  d energy / d (x, y, angle) (nullable)
 *   cand   [configs]       uint32 pairs with centre distance^2 < 2 (nullable)
 * The energy model is the reference's total_cached (seeded.cu:148-162) with
 * pair_cached (seeded.cu:41-65) and boundary (seeded.cu:96-113); the gradient
 * is the sum over pairs of d pair / d square plus the boundary gradient, as
 * the reference's polish assembles it (seeded.cu:637-650).  `threads`
 * selects the kernel: 0 = chosen by n; 32, 64, 128 or 256 = one CTA of that
 * width per configuration; -2, -4 or -8 = one warp per configuration with
 * that many warps per CTA (n <= 256). */
int sqs_sat_energy(sqs_ctx* ctx, int configs, int n, const float* xya, const float* side,
                   float* energy, float* grad, uint32_t* cand, int threads);
/* The same with host buffers: copies in, launches, copies out, synchronises. */
int sqs_sat_energy_host(sqs_ctx* ctx, int configs, int n, const float* xya, const float* side,
                        float* energy, float* grad, uint32_t* cand);

/* ---------------------------------------------------- interval certifier */
#define SQS_CERT_ROUNDTRIP 1 /* re-read every literal through a double first */

typedef struct sqs_verdict {
    int32_t ok;        /* 1 accepted, 0 rejected                              */
    int32_t n;
    double score;      /* max(0, L/sqrt(n) - 1), or the grid penalty if rejected */
    char L[80];        /* side to 50 decimals when accepted, else ""           */
    char reason[112];  /* "ok" or the reference certifier's rejection reason    */
} sqs_verdict;

/* Certify `count` packings.  Packing p has n_of[p] expected squares and rows
 * row_start[p] .. row_start[p+1]-1; row r has square id square_id[r] (NULL:
 * the row's position within its packing) and three decimal literals x, y,
 * angle (radians) at text[lit_off[3r+k] .. lit_off[3r+k+1]), k = 0, 1, 2.
 * Every verdict, reason, score and 50-decimal side equals the reference
 * certifier's evaluate_single_puzzle (certifier.cpp:738-912) on the same
 * strings; SQS_CERT_ROUNDTRIP applies its --roundtrip literal transform
 * (certifier.cpp:914-929, main :1002-1006) first.  Replaces the `certifier`
 * process (certifier.cpp:933-1077) and the Python gate core.certify /
 * core.evaluate (core.py:52-62) for whole batches. */
int sqs_certify_batch(sqs_ctx* ctx, int count, const int32_t* n_of, const int64_t* row_start,
                      const int32_t* square_id, const char* text, const int64_t* lit_off, int flags,
                      sqs_verdict* out);

/* Allocation-free form of sqs_certify_batch, for callers that cannot
 * allocate GPU memory while they run: a host that hands all device memory to
 * its own pool at start-up, or a latency-critical loop that forbids
 * allocation once it runs.  No counterpart in the reference, which always
 * certifies on the CPU.  Same arguments, results and errors as
 * sqs_certify_batch, but it calls no cudaMalloc, cudaFree or other allocating
 * routine: all device scratch is one static array of about 7.6 MiB that
 * every device loading the library holds until process exit, and host
 * staging is static too.  Limits per call: 4,096 packings, 16,384 squares,
 * 2 MiB of literal text (and, with SQS_CERT_ROUNDTRIP, literals under 4,096
 * bytes); larger calls fail with SQS_EINVAL.
 * Set-up: the first call on a device looks up the array's device address
 * (which, under CUDA's lazy module loading, is when the driver loads the
 * module holding it), uploads constants and launches each kernel of the path
 * once with nothing to do (loading it and letting the driver size the local
 * memory its stack needs).  A call with count = 0 does only this set-up.
 * Make that first call at start-up, before a pool takes the device's memory
 * and before any stream capture; afterwards calls allocate nothing.
 * The scratch keeps the last call's contents (what must start at zero is
 * cleared on entry).  Every call in the process shares it -- calls from
 * several threads, contexts or devices -- so calls must not overlap; one
 * that would overlap another call still running fails with SQS_EBUSY. */
int sqs_certify_batch_static(sqs_ctx* ctx, int count, const int32_t* n_of, const int64_t* row_start,
                             const int32_t* square_id, const char* text, const int64_t* lit_off, int flags,
                             sqs_verdict* out);

/* ------------------------------------------------ annealing + polish */
/* One anneal-and-certify job: parallel tempering of n unit squares in a
 * container that shrinks after every new best state.  The job's whole
 * trajectory is a function of its inputs and `seed` alone (counter-based
 * RNG), so it is the same alone or batched with other jobs. */
typedef struct sqs_job {
    int32_t n;               /* squares, 1..1000                                  */
    int32_t replicas;        /* temperature rungs, 1..64                          */
    int32_t sweeps;          /* budget in sweeps (one sweep = n proposals per
                                replica); negative: -sweeps proposals per replica */
    int32_t exchange_every;  /* sweeps between checkpoints (best-state search,
                                shrink, replica exchange); negative: every
                                -exchange_every proposals per replica, as the
                                reference checkpoints after every epoch of
                                `steps` proposals; 0 = chosen by the autotuner
                                (needs SQS_JOB_AUTOTUNE)                          */
    int32_t polish_iters;    /* FP64 gradient-polish iterations on the best state */
    int32_t flags;           /* SQS_JOB_* bits, 0 = fixed default launch shape    */
    double L0;               /* initial container side                            */
    double tmin, tmax;       /* geometric temperature ladder                      */
    double sigma_xy;         /* proposal std-dev of a centre coordinate           */
    double sigma_a;          /* proposal std-dev of the angle (radians)           */
    double shrink;           /* relative shrink of the side after each improvement*/
    uint64_t seed;
    const double* xya;       /* initial state, n rows of (x, y, angle), host      */
    const double* xya_rep;   /* optional: replicas * n rows, each replica's own
                                start (e.g. from sqs_portfolio); NULL: every
                                replica starts from xya                          */
} sqs_job;

/* Launch shape, cell side and (when the job leaves it at 0) exchange
 * interval from the autotuner (sqs_autotune) instead of the fixed default:
 * the smallest cluster that fits, cells of side 1.59.  Shape and cell side
 * do not change a job's trajectory (energies are exact fixed-point sums, the
 * quench sums each square's gradient in one thread); only a move rejected
 * because its target cell was full can, and sqs_job_result.overflows counts
 * those. */
#define SQS_JOB_AUTOTUNE 1
/* Move-set options, each a counterpart of the reference search's moves:
 *  ADAPT       steps drawn uniform in +-sigma per coordinate and angle (the
 *              reference's draws; Gaussian of deviation sigma without it),
 *              step size per replica scaled by its rung (0.15 .. 2 x sigma
 *              from the coldest to the hottest rung), by an adaptation factor
 *              that every 16 proposals moves toward 25% acceptance
 *              (x exp((rate - 0.25) / 2), kept in [0.1, 4]), by 3.5 on every
 *              16th proposal, and a cooling cycle of 200 exchange rounds that
 *              scales temperatures by 0.002^(k/199) and steps by its square
 *              root (seeded.cu:493-494, 506-507, 614-618);
 *  COLLECTIVE  6 proposals in 7 move a set of squares around the drawn one:
 *              its row, its column, a disc of radius^2 2.5, its orientation
 *              class, its diagonal strips, or all tilted squares, translated
 *              (and rotated about it for the disc and the class), judged on
 *              the full energy (seeded.cu:547-613);
 *  KICK        at every exchange round an overlapped replica has its squares
 *              jittered (more where their energy is higher) and, every other
 *              round, its worst square moved to the emptiest point of an 8 x 8
 *              probe grid (seeded.cu:721-778).
 * All draws are counter-based, so a job stays reproducible and independent
 * of batching, slicing and launch shape. */
#define SQS_JOB_ADAPT 2
#define SQS_JOB_COLLECTIVE 4
#define SQS_JOB_KICK 8
/* Evaluate proposals strictly one at a time.  Without move-set options a
 * replica's warp evaluates two consecutive proposals at once, one per
 * half-warp, against the same state, and evaluates the second again when the
 * first was accepted and moved something the second read (the same square,
 * or a square or cell list inside its 3 x 3 cell block).  Energies are exact
 * integers, so the trajectory is the one-at-a-time trajectory bit for bit;
 * this flag changes only the time taken, and lets a caller check that. */
#define SQS_JOB_SERIAL 16
/* Quench every replica, not only the coldest, at each exchange round: the
 * counterpart of the reference search's per-epoch gradient polish of every
 * chain (seeded.cu:621-713).  Costs one quench per replica per round. */
#define SQS_JOB_QUENCH_ALL 32
/* Dilation-certify every replica at each checkpoint, not only those whose
 * overlap energy is below 1e-4: the reference search measures every chain's
 * certified side after its polish, whatever its overlap (seeded.cu:716-720,
 * device_certified_side :175-226; a dilation above 1.008 still rejects).
 * Costs one FP64 side measurement per replica per checkpoint. */
#define SQS_JOB_CERT_ALL 64
/* Checkpoint quench budget, k = 1..127: up to 16 k conjugate-gradient
 * iterations per quench, ending only at zero overlap or a zero gradient (a
 * line search that finds no lower energy drops the direction, halves the
 * step and goes on), as the reference's per-epoch polish runs its iterations
 * uninterrupted (seeded.cu:621-713).  k = 0: 64 iterations, also ending
 * at a line search without a gain or after three accepted steps in a row
 * that each gained less than 0.1%. */
#define SQS_JOB_QUENCH_STEPS(k) ((int32_t)(k) << 24)
/* The reference search's target-side ladder (seeded.cu:474-481, 908-943): from
 * the first proposal every rung anneals in its own container below the best
 * side B found so far (the initial side before the first certificate; only
 * a certified side below the initial one counts, as the reference's chain
 * bests start at the seed's side):
 * side max(sqrt n + 1e-6, B (1 - shrink m)) with m the reference's offsets
 * {0.02, 0.1, 0.4, 1, 2.5, 5, 10, 20} for the rung's place in its ladder.  A
 * new certified best becomes B (no further factor), every ladder's head rung
 * (and, after a gain above 5e-4, every rung of ladder 0) restarts from the
 * new best state scaled into its side, and replicas exchange only at
 * checkpoints without a new best.  Energies are measured in each replica's
 * own side. */
#define SQS_JOB_TARGETS 128
/* Split the job's rungs into l ladders of replicas / l rungs each (l = 1..15,
 * dividing replicas): temperatures, step scales and target offsets run over a
 * ladder's rungs, and exchange pairs neighbours within a ladder, as the
 * reference runs its chains as ladders of 8 (seeded.cu:493, 791-817); the
 * ladders share the job's best side.  0 or 1: one ladder. */
#define SQS_JOB_LADDERS(l) ((int32_t)(l) << 20)
/* Pin the launch shape instead of SQS_JOB_AUTOTUNE: a cluster of `cs` CTAs (1..16; it must
 * divide the replica count and fit) and cell side index k (0: 1.59, 1: 1.75,
 * 2: 1.95, 3: 2.2).  Same trajectory as any other shape (see above). */
#define SQS_JOB_CLUSTER(cs) ((int32_t)(cs) << 8)
#define SQS_JOB_CELL(k) ((int32_t)(k) << 16)

typedef struct sqs_job_result {
    int32_t status;          /* 0 ok; < 0 job error (see reason)                  */
    int32_t certified;       /* the interval certifier accepted the packing      */
    int32_t shrinks, improvements, sweeps_done, replicas;
    int32_t cluster_ctas;    /* CTAs per job the job ran on                       */
    int32_t replicas_per_cta;/* replicas (warps) per CTA                          */
    int32_t exchange_every;  /* sweeps between exchange rounds it ran with        */
    int32_t overflows;       /* moves rejected because the target cell was full  */
    double cell_side;        /* minimum cell side of its cell lists               */
    double L_cert;           /* FP64 dilation-certified side of the best state    */
    double L_polished;       /* the same after the gradient polish                */
    double dilation;         /* centre dilation under which the packing certified*/
    double score;            /* max(0, L/sqrt(n) - 1) of the certified side       */
    int64_t proposals, accepted, exchange_attempts, exchange_accepts;
    double device_ms;        /* device time of this call (all jobs)               */
    char L[80];              /* certified side, 50 decimals ("" if none)          */
    char reason[112];
} sqs_job_result;

/* Anneal, polish and certify `njobs` jobs in persistent batched launches
 * (one thread-block cluster per job, one warp per replica) and return each
 * job's best packing in xya_out[j] (caller buffer of n*3 doubles; centres
 * after the certifying dilation, angles in [0, pi/2)).  Replaces the
 * reference's `packing` / `seeded` search programs (packing.cu:768-868,
 * seeded.cu:831-983) and its certified_candidate dilation ladder
 * (demo.py:25-40).  slice_sweeps > 0 runs the jobs in slices of that many
 * sweeps (state kept resident in HBM between slices); 0 = one slice.  With
 * three or more slices the slice loop is captured once as a CUDA graph (one
 * launch per cluster shape) and replayed.  Jobs flagged SQS_JOB_AUTOTUNE are
 * tuned for latency when njobs == 1, for throughput otherwise. */
int sqs_anneal_batch(sqs_ctx* ctx, const sqs_job* jobs, int njobs, int slice_sweeps, double* const* xya_out,
                     sqs_job_result* out);

/* Each replica's final state, for checking the annealer against an FP64
 * recomputation.  Caller buffers sized by the job's replicas R and n; any of
 * them may be NULL. */
typedef struct sqs_replica_trace {
    float* xya;              /* R * n * 3: each replica's final (x, y, angle), FP32 as annealed */
    double* energy;          /* R: the annealer's running energy of each replica (walls + pairs:
                                its exact fixed-point sum, in energy units)                        */
    double* energy_full;     /* R: the same recomputed from scratch on the final state            */
    double* L_cert;          /* R: FP64 dilation-certified side of the final state, by the device
                                function the checkpoints use (1e9: dilation above 1.008)          */
    double* dilation;        /* R: that dilation                                                   */
    float* side;             /* R: the container side each energy is measured in                  */
    float* temperature;      /* R: temperature of each replica's next proposal (rung x cooling)  */
    float* step_scale;       /* R: step scale of its next proposal, in units of sigma (1 without
                                SQS_JOB_ADAPT)                                                     */
    int32_t* rung;           /* R: temperature index of each replica                               */
    int32_t exchange_rounds; /* out: exchange rounds the job completed                             */
    int32_t cells_ok;        /* out: every final state fitted its cell list                        */
} sqs_replica_trace;

/* sqs_anneal_batch, then each job's replicas read back into trace[j] (one
 * record per job): their final states, running energies and the checks
 * above, measured after the timed region (result.device_ms excludes it).
 * The reference's counterpart is its device self-tests, which compare the
 * search's running FP32 energy with a host FP64 sum (cuda/tests/
 * globaltest.cu:21-49). */
int sqs_anneal_batch_trace(sqs_ctx* ctx, const sqs_job* jobs, int njobs, int slice_sweeps, double* const* xya_out,
                           sqs_job_result* out, sqs_replica_trace* trace);

/* FP64 energy (walls + sum over pairs of the squared SAT penetration) and
 * its gradient of `count` packings, one CTA each, all pairs: the FP64
 * recompute of a candidate state.  Packing k has n_of[k] rows (1..1000) of
 * (x, y, angle) in xya, back to back, and container side side[k]; energy[k]
 * and, when grad is not NULL, grad (the layout of xya) = d energy /
 * d (x, y, angle).  The pair term is the reference's pair_cached
 * (seeded.cu:41-65), the gradient its polish's pair_cached_smooth
 * (seeded.cu:67-90) with the smooth wall derivative (seeded.cu:96-113),
 * summed per square as seeded.cu:637-650 does; cos and sin are taken of the
 * angles as given.  Replaces the reference's FP64 total_cached
 * (seeded.cu:148-162) and its polish gradient. */
int sqs_energy_fp64(sqs_ctx* ctx, int count, const int32_t* n_of, const double* xya, const double* side,
                    double* energy, double* grad);

/* Initial states of `chains` search chains (out: chains * n rows of x, y,
 * angle), the reference's structured portfolio (build_portfolio,
 * seeded.cu:233-425): by chain b's group b % 8 within its ladder b / 8, the
 * seed, one of up to 64 corner-triangle + 45-degree-band topologies that fit
 * n to n + 4 squares in a side within [sqrt n - 0.05, L + 0.15], a corner
 * grid with tilted edge rows, or corner anchors with a rotated grid.
 * structured = 0 copies the seed to every chain.  jitter != 0 then applies
 * the per-chain jitter of structured_init (seeded.cu:427-451: none for group
 * 0, 1e-4 * 100^u for group 1, 0.03 otherwise) from rng_seed with this
 * library's generator.  Host only; the layouts before the jitter equal the
 * reference's bit for bit.  The chains of ladder k are the replicas of an
 * 8-replica job (sqs_job.xya_rep). */
int sqs_portfolio(int n, double L, const double* seed_xya, int chains, int structured, uint64_t rng_seed, int jitter,
                  double* out);

/* FP64 gradient polish of `count` packings, one CTA each, all pairs.
 * Packing k has n_of[k] rows (1..1000) of (x, y, angle) in xya, packings
 * back to back; the polished packings go to xya_out (same layout; may equal
 * xya), translated so the bounding box of the certifying dilation starts at
 * the origin.  The incumbent is the input's FP64 dilation-certified side
 * (seeded.cu:175-226: every close pair separated once the centres are
 * scaled by lambda <= 1.008); an input too overlapped for that first
 * descends its overlap energy inside its own bounding box (half the budget)
 * and, if overlaps remain, with its centres spread by lambda (at most 1.5x)
 * in a box scaled alike.  Each attempt
 * compresses the incumbent by 1 - delta, descends the squared-penetration
 * energy (pair_cached_smooth, seeded.cu:67-90) with a backtracking line
 * search, and keeps the result when its certified side is smaller; delta
 * shrinks after a failed attempt; `iters` bounds the gradient steps.
 * Replaces the reference's polish (cuda/polish.py:67-107, SLSQP on the
 * CPU for n <= 50) and its device polish of every chain (seeded.cu:621-713).
 * The side is the FP64 dilation bound; the interval certifier's verdict is
 * sqs_certify_batch's (polish.certify_q applies the dilation ladder). */
typedef struct sqs_polish_result {
    double L_in;             /* certified side of the input (1e30: none)       */
    double L_out;            /* the same after the polish (1e30: none)         */
    int32_t iterations;      /* gradient steps used                            */
    int32_t improved;        /* L_out < L_in                                   */
} sqs_polish_result;
int sqs_polish_batch(sqs_ctx* ctx, int count, const int32_t* n_of, const double* xya, int iters, double* xya_out,
                     sqs_polish_result* out);

/* Autotuner of the batched annealer's launch: times the job's own state on
 * every launch shape that fits (cluster size x replicas per CTA) and cell
 * sides 1.59 .. 2.2, with the job copied to fill one wave of the GPU
 * (throughput) or alone (latency), then, when job->exchange_every is 0, the
 * exchange interval: the smallest of 1, 2, 5, 10, 20, 50, 100 sweeps whose
 * checkpoint costs at most 5% of the sweeps between.  Choices are cached per
 * process by (n rounded to a quarter octave, replicas, mode); a cached class
 * returns at once (trials = 0).  The reference tunes its search launches
 * offline by sweeping configurations in separate runs (cuda/autotune.py). */
typedef struct sqs_tuning {
    int32_t cluster_ctas;      /* CTAs per job                                  */
    int32_t replicas_per_cta;  /* warps per CTA, one replica each               */
    int32_t exchange_every;    /* the job's, or the tuned one when it was 0     */
    int32_t trials;            /* timed launches (0: answered from the cache)  */
    double cell_side;          /* minimum cell side                             */
    double us_per_sweep;       /* device time per sweep of the chosen shape     */
} sqs_tuning;
#define SQS_TUNE_LATENCY 1     /* time the job alone instead of a full wave     */
int sqs_autotune(sqs_ctx* ctx, const sqs_job* job, int mode, sqs_tuning* out);

/* ------------------------------------------------------------- serving */
/* Continuous-batching request loop for anneal-and-certify jobs on one GPU.
 * Jobs are admitted while a job slot is free and their state (replicas,
 * scratch, best packing) fits an HBM arena of `hbm_bytes`.  Each job runs in
 * slices of `slice_sweeps` sweeps (slice_sweeps < 0: about -slice_sweeps
 * proposals per replica -- ceil(-slice_sweeps / n) sweeps rounded up to
 * whole exchange intervals -- so a slice takes about the same time for small
 * and large jobs), launched together with the other idle jobs of its cluster
 * shape as soon as its previous slice ends, its state resident between
 * slices.  Finished jobs are polished, certified and retired by the server's
 * own thread, and queued jobs take their place.  Each job's result equals
 * its sqs_anneal_batch result.
 * Replaces one-search-process-per-job campaigns (scheduler.run_gpu,
 * cuda/scheduler.py:80-89) and their VRAM-budgeted worker admission
 * (cpp_loop.concurrency, cuda/cpp_loop.py:41-45). */
typedef struct sqs_server sqs_server;
int sqs_server_create(sqs_ctx* ctx, size_t hbm_bytes, int max_active, int slice_sweeps, sqs_server** out);
int sqs_server_destroy(sqs_server* server);
/* Queue a job (the job and its initial state are copied). */
int sqs_server_submit(sqs_server* server, const sqs_job* job, int64_t* id);
/* One round of the loop: admit queued jobs; collect the slices that have
 * finished; start the next slice of every idle job (one launch per cluster
 * shape, each on its own stream, so slices of different jobs start and end
 * independently); hand the jobs whose budget is spent to the server's
 * retirement thread, which polishes, certifies and retires them while the
 * slices run.  When there is nothing to do it waits up to 2 ms for a slice
 * or a retirement to finish.  *in_flight = queued + running + retiring.
 * Server calls come from one thread at a time, as for a context. */
int sqs_server_step(sqs_server* server, int* in_flight);
/* 1 and the result (and n*3 packing into xya_out when certified) once the
 * job is done -- the job is then forgotten; 0 while it is queued or running;
 * SQS_ENOTFOUND for an unknown id. */
int sqs_server_poll(sqs_server* server, int64_t id, sqs_job_result* out, double* xya_out);
/* Withdraw a queued job now, or a running one when its slice in flight ends
 * (it is retired uncertified by the step that collects that slice). */
int sqs_server_cancel(sqs_server* server, int64_t id);
int sqs_server_info(sqs_server* server, int* queued, int* active, size_t* hbm_used);
/* Counters since the server's creation: steps, slice launches, jobs
 * admitted and retired, and host wall seconds -- of the steps' admission
 * (state upload), of harvesting finished slices and launching new ones, of
 * waiting when there was nothing else to do, and of retirement (polish,
 * rescue, certification), which runs on the server's own thread while the
 * steps go on; polish_s and certify_s are the polish (launch to results on
 * the host) and the certification ladder within retire_s. */
typedef struct sqs_server_stats {
    int64_t steps, slices, admitted, retired;
    double admit_s, launch_s, retire_s, wait_s, polish_s, certify_s;
} sqs_server_stats;
int sqs_server_get_stats(sqs_server* server, sqs_server_stats* out);

#ifdef __cplusplus
}
#endif
#endif /* SQS_H */
