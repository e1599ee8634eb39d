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
/* Kernel launches this context issued since creation (all of libsqs's own
 * kernels; library copies/memsets are not counted). */
int64_t sqs_launch_count(sqs_ctx* ctx);

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
 * the reference's polish assembles it (seeded.cu:637-650).  `threads` is the
 * CTA width (32, 64, 128 or 256; 0 = chosen by n). */
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

#ifdef __cplusplus
}
#endif
#endif /* SQS_H */
