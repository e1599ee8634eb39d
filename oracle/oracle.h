/* TEST INFRASTRUCTURE ONLY -- declarations of the CPU oracle (liboracle.so).
 * Loaded by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg
 * as the checker of the CUDA path; never linked by the product. */
#ifndef SQS_ORACLE_H
#define SQS_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
/* sat_oracle.c: FP64 SAT pair energy, wall penalty and total energy */
double sqo_pair_cached(const double p[3], const double q[3], double c, double s,
                       double d, double t, double* grad, int smooth);
double sqo_pair(const double p[3], const double q[3], double* grad);
double sqo_boundary(const double p[3], double L, double* g);
double sqo_total(int n, double L, const double* xya, double* grad, int64_t* cand);
double sqo_total_smooth(int n, double L, const double* xya, double* grad);
int sqo_total_batch(int configs, int n, const double* xya, const double* L,
                    double* energy, double* grad, int64_t* cand, int threads);
/* ptsa_oracle.c: dilation-certified side of a state and the CPU PT-SA */
double sqo_certified_side(int n, const double* xya, double* best_out, double* lam_out);
typedef struct sqo_job {
    int n, replicas, sweeps, exchange_every;
    double L0, tmin, tmax, sigma_xy, sigma_a, shrink;
    uint64_t seed;
    const double* xya;
} sqo_job;
typedef struct sqo_job_out {
    double best_L;
    long long proposals, accepted, xatt, xacc;
    int shrinks, pad;
} sqo_job_out;
int sqo_ptsa_batch(int njobs, const sqo_job* jobs, sqo_job_out* out, int threads);
/* certify_oracle.cpp: interval certifier of one packing */
int sqo_certify(int n, int rows, const int* sid, const char* const* xs, const char* const* ys,
                const char* const* as, char* L_out, int L_cap, char* reason_out, int reason_cap,
                double* score);
void sqo_roundtrip(const char* s, char* out, int cap);
#ifdef __cplusplus
}
#endif
#endif
