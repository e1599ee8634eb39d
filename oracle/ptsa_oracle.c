/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle for the FP64 best-state recompute.
 *
 * Loaded only by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg as the checker of the CUDA path.
 *
 * sqo_certified_side restates device_certified_side (seeded.cu:175-226,
 * packing.cu:254-297): the smallest centre dilation lambda >= 1 that opens a
 * tau = 2.6e-8 gap along the best SAT axis of every close pair (centre
 * distance^2 < 2.05), rejection when lambda > 1.008, then the side of the
 * bounding box of the lambda-scaled squares.  The state written to best_out
 * is translated so its box starts at the origin, angles wrapped to [0, pi/2)
 * (wrap_angle, seeded.cu:28-33).
 */
#include <math.h>
#include <stddef.h>
#include "oracle.h"

static double wrap_quarter(double a) {
    const double q = 1.57079632679489661923;
    a = fmod(a, q);
    if (a < 0.0) a += q;
    return a;
}

double sqo_certified_side(int n, const double* xya, double* best_out, double* lam_out) {
    const double tau = 2.6e-8;
    double lam = 1.0;
    for (int i = 0; i < n; i++) {
        double xi = xya[3 * i], yi = xya[3 * i + 1];
        double ci = cos(xya[3 * i + 2]), si = sin(xya[3 * i + 2]);
        for (int j = i + 1; j < n; j++) {
            double dx = xi - xya[3 * j], dy = yi - xya[3 * j + 1];
            if (dx * dx + dy * dy >= 2.05) continue;
            double cj = cos(xya[3 * j + 2]), sj = sin(xya[3 * j + 2]);
            double c12 = fabs(ci * cj + si * sj), s12 = fabs(-si * cj + ci * sj);
            double r = 0.5 + 0.5 * (c12 + s12);
            double v1 = fabs(dx * ci + dy * si), v2 = fabs(-dx * si + dy * ci);
            double v3 = fabs(dx * cj + dy * sj), v4 = fabs(-dx * sj + dy * cj);
            double vmax = fmax(fmax(v1, v2), fmax(v3, v4));
            double req = (vmax > 1e-12) ? ((r + tau) / vmax) : 1e9;
            if (req > lam) lam = req;
        }
    }
    if (lam_out) *lam_out = lam;
    if (lam > 1.008) return 1e9;
    double x0 = 1e9, x1 = -1e9, y0 = 1e9, y1 = -1e9;
    for (int i = 0; i < n; i++) {
        double x = xya[3 * i] * lam, y = xya[3 * i + 1] * lam;
        double c = cos(xya[3 * i + 2]), s = sin(xya[3 * i + 2]);
        double r = 0.5 * (fabs(c) + fabs(s));
        if (x - r < x0) x0 = x - r;
        if (x + r > x1) x1 = x + r;
        if (y - r < y0) y0 = y - r;
        if (y + r > y1) y1 = y + r;
    }
    double L = fmax(x1 - x0, y1 - y0);
    if (best_out) {
        for (int i = 0; i < n; i++) {
            best_out[3 * i] = xya[3 * i] * lam - x0;
            best_out[3 * i + 1] = xya[3 * i + 1] * lam - y0;
            best_out[3 * i + 2] = wrap_quarter(xya[3 * i + 2]);
        }
    }
    return L;
}

/*
 * CPU parallel-tempering annealer: the CPU baseline of the plain and batched
 * search workloads (timed by bench.py's cpu_baseline leg only).
 *
 * The reference has no CPU search; this restates its per-proposal scheme
 * (seeded.cu:454-546, single-square moves): pick a square, displace its
 * centre and angle, evaluate the FP64 energy change against every other
 * square (pair_cached seeded.cu:41-65, boundary seeded.cu:96-113: O(n) per
 * proposal), accept by Metropolis at the replica's rung temperature.  Rungs
 * form a geometric ladder tmin..tmax; every `exchange_every` sweeps the
 * replicas of neighbouring rungs swap by the exchange rule of swap_replicas
 * (seeded.cu:791-817, alternating parity), and every replica whose energy is
 * below 1e-4 has its dilation-certified side measured (sqo_certified_side);
 * a new best side shrinks the container by the factor (1 - shrink) and
 * rescales every replica into it (the host shrink loop, seeded.cu:908-943).
 * Steps are Gaussian (sigma_xy clamped to +-0.12, sigma_a), centres kept in
 * [0.5, L - 0.5], angles wrapped to [0, pi/2), as the GPU annealer draws them.
 * Jobs run in parallel on `threads` host threads; each job is sequential.
 */
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    uint64_t s[4];
} sqo_rng;

static uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
static uint64_t splitmix64(uint64_t* x) {
    uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static void rng_seed(sqo_rng* r, uint64_t seed) {
    for (int k = 0; k < 4; ++k) r->s[k] = splitmix64(&seed);
}
static uint64_t rng_next(sqo_rng* r) { /* xoshiro256** */
    uint64_t* s = r->s;
    const uint64_t out = rotl64(s[1] * 5, 7) * 9, t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl64(s[3], 45);
    return out;
}
static double rng_u01(sqo_rng* r) { return ((double)(rng_next(r) >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
static double rng_gauss(sqo_rng* r) {
    return sqrt(-2.0 * log(rng_u01(r))) * cos(6.283185307179586 * rng_u01(r));
}

/* energy of square i of state q (n x 3, trig cached) against all others, plus its wall term */
static double square_energy(int n, const double* q, const double* cs, int i, const double* p, double c, double s,
                            double L) {
    double e = sqo_boundary(p, L, NULL);
    for (int j = 0; j < n; ++j) {
        if (j == i) continue;
        e += sqo_pair_cached(p, q + 3 * j, c, s, cs[2 * j], cs[2 * j + 1], NULL, 0);
    }
    return e;
}

static double state_energy(int n, const double* q, const double* cs, double L) {
    double e = 0.0;
    for (int i = 0; i < n; ++i) {
        e += sqo_boundary(q + 3 * i, L, NULL);
        for (int j = i + 1; j < n; ++j)
            e += sqo_pair_cached(q + 3 * i, q + 3 * j, cs[2 * i], cs[2 * i + 1], cs[2 * j], cs[2 * j + 1], NULL, 0);
    }
    return e;
}

static void run_job(const sqo_job* J, sqo_job_out* o) {
    const int n = J->n, R = J->replicas;
    double* q = (double*)malloc(sizeof(double) * 3 * (size_t)n * R);
    double* cs = (double*)malloc(sizeof(double) * 2 * (size_t)n * R);
    double* E = (double*)malloc(sizeof(double) * R);
    double* T = (double*)malloc(sizeof(double) * R);
    int* rung = (int*)malloc(sizeof(int) * R);
    int* holder = (int*)malloc(sizeof(int) * R);
    sqo_rng* rng = (sqo_rng*)malloc(sizeof(sqo_rng) * (R + 1));
    double L = J->L0;
    memset(o, 0, sizeof *o);
    o->best_L = 1e30;
    for (int r = 0; r < R; ++r) {
        for (int i = 0; i < n; ++i) {
            double* p = q + 3 * ((size_t)r * n + i);
            p[0] = J->xya[3 * i];
            p[1] = J->xya[3 * i + 1];
            p[2] = wrap_quarter(J->xya[3 * i + 2]);
            cs[2 * ((size_t)r * n + i)] = cos(p[2]);
            cs[2 * ((size_t)r * n + i) + 1] = sin(p[2]);
        }
        E[r] = state_energy(n, q + 3 * (size_t)r * n, cs + 2 * (size_t)r * n, L);
        T[r] = R > 1 ? exp(log(J->tmin) + (log(J->tmax) - log(J->tmin)) * r / (double)(R - 1)) : J->tmin;
        rung[r] = r;
        rng_seed(&rng[r], J->seed ^ (0xA24BAED4963EE407ull * (uint64_t)(r + 1)));
    }
    rng_seed(&rng[R], J->seed ^ 0x9FB21C651E98DF25ull);
    double* bestq = (double*)malloc(sizeof(double) * 3 * (size_t)n);
    int xround = 0;
    for (int sweep = 0; sweep < J->sweeps; ++sweep) {
        for (int r = 0; r < R; ++r) {
            double* Q = q + 3 * (size_t)r * n;
            double* C = cs + 2 * (size_t)r * n;
            const double invT = 1.0 / T[rung[r]];
            for (int k = 0; k < n; ++k) {
                sqo_rng* g = &rng[r];
                const int i = (int)((rng_next(g) >> 32) * (uint64_t)n >> 32);
                double dx = J->sigma_xy * rng_gauss(g), dy = J->sigma_xy * rng_gauss(g);
                dx = fmin(0.12, fmax(-0.12, dx));
                dy = fmin(0.12, fmax(-0.12, dy));
                const double da = J->sigma_a * rng_gauss(g);
                const double* P = Q + 3 * i;
                double np[3];
                np[0] = fmin(fmax(P[0], L - 0.5), fmax(fmin(P[0], 0.5), P[0] + dx));
                np[1] = fmin(fmax(P[1], L - 0.5), fmax(fmin(P[1], 0.5), P[1] + dy));
                np[2] = wrap_quarter(P[2] + da);
                const double nc = cos(np[2]), ns = sin(np[2]);
                const double de = square_energy(n, Q, C, i, np, nc, ns, L) -
                                  square_energy(n, Q, C, i, P, C[2 * i], C[2 * i + 1], L);
                o->proposals++;
                if (de <= 0.0 || rng_u01(g) < exp(-de * invT)) {
                    o->accepted++;
                    E[r] += de;
                    Q[3 * i] = np[0];
                    Q[3 * i + 1] = np[1];
                    Q[3 * i + 2] = np[2];
                    C[2 * i] = nc;
                    C[2 * i + 1] = ns;
                }
            }
        }
        if ((sweep + 1) % J->exchange_every != 0 && sweep + 1 != J->sweeps) continue;
        /* best-state search and shrink */
        double newL = L;
        for (int r = 0; r < R; ++r) {
            if (E[r] >= 1e-4) continue;
            double lam = 0.0;
            const double Lc = sqo_certified_side(n, q + 3 * (size_t)r * n, bestq, &lam);
            if (Lc < o->best_L) {
                o->best_L = Lc;
                newL = fmin(newL, Lc * (1.0 - J->shrink));
            }
        }
        if (newL < L) {
            const double f = newL / L;
            L = newL;
            o->shrinks++;
            for (int r = 0; r < R; ++r) {
                double* Q = q + 3 * (size_t)r * n;
                for (int i = 0; i < n; ++i) {
                    Q[3 * i] *= f;
                    Q[3 * i + 1] *= f;
                }
                E[r] = state_energy(n, Q, cs + 2 * (size_t)r * n, L);
            }
        }
        /* neighbouring-rung exchange, alternating parity */
        for (int r = 0; r < R; ++r) holder[rung[r]] = r;
        for (int k = xround & 1; k + 1 < R; k += 2) {
            const int a = holder[k], b = holder[k + 1];
            const double d = (1.0 / T[k] - 1.0 / T[k + 1]) * (E[a] - E[b]);
            o->xatt++;
            if (d >= 0.0 || rng_u01(&rng[R]) < exp(d)) {
                o->xacc++;
                rung[a] = k + 1;
                rung[b] = k;
                holder[k] = b;
                holder[k + 1] = a;
            }
        }
        xround++;
    }
    free(bestq);
    free(q);
    free(cs);
    free(E);
    free(T);
    free(rung);
    free(holder);
    free(rng);
}

typedef struct {
    int njobs;
    const sqo_job* jobs;
    sqo_job_out* out;
    int next;
    pthread_mutex_t mu;
} ptsa_pool;

static void* ptsa_worker(void* arg) {
    ptsa_pool* P = (ptsa_pool*)arg;
    for (;;) {
        pthread_mutex_lock(&P->mu);
        const int j = P->next++;
        pthread_mutex_unlock(&P->mu);
        if (j >= P->njobs) return NULL;
        run_job(&P->jobs[j], &P->out[j]);
    }
}

int sqo_ptsa_batch(int njobs, const sqo_job* jobs, sqo_job_out* out, int threads) {
    if (njobs <= 0) return 0;
    if (threads < 1) threads = 1;
    if (threads > njobs) threads = njobs;
    ptsa_pool P = {njobs, jobs, out, 0, PTHREAD_MUTEX_INITIALIZER};
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)threads);
    for (int t = 0; t < threads; ++t) pthread_create(&th[t], NULL, ptsa_worker, &P);
    for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
    free(th);
    return threads;
}
