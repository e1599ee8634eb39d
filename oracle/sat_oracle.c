/*
 * TEST INFRASTRUCTURE ONLY -- the CPU oracle for the SAT overlap energy.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load
 * this file's shared library, and only as the checker of the CUDA path.
 * Nothing in the product links it.
 *
 * A plain-C FP64 restatement of the reference's energy model for n unit
 * squares (x, y, angle) in the container [0, L]^2:
 *
 *   pair energy    seeded.cu:41-65   (pair_cached, gradient of the first square)
 *                  seeded.cu:92-94   (pair: cos/sin taken from the angles)
 *   smooth variant seeded.cu:67-90   (pair_cached_smooth, used by the polish)
 *   wall penalty   seeded.cu:96-113  (boundary, with dr_smooth gradient :36-38)
 *   total energy   seeded.cu:148-162 (total_cached: walls + sum over i<j)
 *
 * Gradient convention (same as the reference): d pair(p,q) / d p.  The full
 * gradient of the total energy for square i is d boundary_i + sum_{j != i}
 * d pair(p_i, p_j) / d p_i, which is how the reference's polish builds it
 * (seeded.cu:637-650).
 *
 * Parity of this file is pinned by tests against the reference's own
 * host-callable pair()/boundary() compiled from seeded.cu into oracle/_ref.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static inline double sgn(double x) { return (double)((x > 0) - (x < 0)); }
static inline double sgn_smooth(double x) {
    return (fabs(x) > 1e-6) ? ((x >= 0.0) ? 1.0 : -1.0) : 0.0;
}
static inline double dr_smooth(double c, double s) {
    return 0.5 * (-sgn_smooth(c) * s + sgn_smooth(s) * c);
}

/* Squared SAT penetration of unit squares p, q with cached cos/sin (c,s) of p
 * and (d,t) of q.  0 when d^2 >= 2.000001 or when an axis separates them.
 * smooth != 0 selects the polish variant (seeded.cu:67-90). */
double sqo_pair_cached(const double p[3], const double q[3], double c, double s,
                       double d, double t, double* grad, int smooth) {
    double dx = q[0] - p[0], dy = q[1] - p[1];
    if (dx * dx + dy * dy >= 2.000001) return 0.0;
    double cd = c * d + s * t, sd = s * d - c * t;
    double radius = 0.5 + 0.5 * (fabs(cd) + fabs(sd));
    double deriv = smooth ? 0.5 * (-sgn_smooth(cd) * sd + sgn_smooth(sd) * cd)
                          : 0.5 * (-sgn(cd) * sd + sgn(sd) * cd);
    double ux[4] = {c, -s, d, -t}, uy[4] = {s, c, t, d};
    double gap = -1e100, gx = 0, gy = 0, ga = 0;
    for (int k = 0; k < 4; k++) {
        double v = dx * ux[k] + dy * uy[k], z = fabs(v) - radius;
        if (z > gap) {
            gap = z;
            double sv = smooth ? ((v >= 0.0) ? 1.0 : -1.0) : sgn(v);
            gx = -sv * ux[k];
            gy = -sv * uy[k];
            ga = -deriv + (k < 2 ? sv * (-dx * uy[k] + dy * ux[k]) : 0.0);
        }
    }
    if (gap >= 0) return 0.0;
    if (grad) {
        grad[0] += 2 * gap * gx;
        grad[1] += 2 * gap * gy;
        grad[2] += 2 * gap * ga;
    }
    return gap * gap;
}

double sqo_pair(const double p[3], const double q[3], double* grad) {
    return sqo_pair_cached(p, q, cos(p[2]), sin(p[2]), cos(q[2]), sin(q[2]), grad, 0);
}

/* Wall penalty sum_k max(0, v_k)^2 with v = (r-x, x+r-L, r-y, y+r-L). */
double sqo_boundary(const double p[3], double L, double* g) {
    double c = cos(p[2]), s = sin(p[2]);
    double r = 0.5 * (fabs(c) + fabs(s));
    double v[4] = {r - p[0], p[0] + r - L, r - p[1], p[1] + r - L}, e = 0;
    double d_r = g ? dr_smooth(c, s) : 0.0;
    for (int k = 0; k < 4; k++) {
        if (v[k] > 0) {
            e += v[k] * v[k];
            if (g) {
                double f = 2 * v[k];
                g[0] += f * (k == 0 ? -1 : k == 1 ? 1 : 0);
                g[1] += f * (k == 2 ? -1 : k == 3 ? 1 : 0);
                g[2] += f * d_r;
            }
        }
    }
    return e;
}

/* Total energy of one configuration (walls + sum_{i<j} pair) and, when grad
 * is given (n*3 doubles, overwritten), its gradient.  *cand (nullable)
 * receives the number of pairs with centre distance^2 < 2. */
static double total_ex(int n, double L, const double* xya, double* grad, int64_t* cand, int smooth);

double sqo_total(int n, double L, const double* xya, double* grad, int64_t* cand) {
    return total_ex(n, L, xya, grad, cand, 0);
}

/* The same with the polish's smooth pair gradient (pair_cached_smooth,
 * seeded.cu:67-90) when smooth != 0; the energy is unchanged. */
double sqo_total_smooth(int n, double L, const double* xya, double* grad) {
    return total_ex(n, L, xya, grad, NULL, 1);
}

static double total_ex(int n, double L, const double* xya, double* grad, int64_t* cand, int smooth) {
    double e = 0.0;
    int64_t pairs = 0;
    if (grad) memset(grad, 0, sizeof(double) * 3 * (size_t)n);
    for (int i = 0; i < n; i++) {
        const double* p = xya + 3 * i;
        double c = cos(p[2]), s = sin(p[2]);
        e += sqo_boundary(p, L, grad ? grad + 3 * i : NULL);
        for (int j = 0; j < n; j++) {
            if (j == i) continue;
            const double* q = xya + 3 * j;
            double dx = q[0] - p[0], dy = q[1] - p[1];
            if (j > i && dx * dx + dy * dy < 2.0) pairs++;
            if (j > i) {
                e += sqo_pair_cached(p, q, c, s, cos(q[2]), sin(q[2]),
                                     grad ? grad + 3 * i : NULL, smooth);
            } else if (grad) {
                sqo_pair_cached(p, q, c, s, cos(q[2]), sin(q[2]), grad + 3 * i, smooth);
            }
        }
    }
    if (cand) *cand = pairs;
    return e;
}

typedef struct {
    int first, last, n;
    const double* xya;
    const double* L;
    double* energy;
    double* grad;
    int64_t* cand;
} sqo_job;

static void* sqo_worker(void* arg) {
    sqo_job* j = (sqo_job*)arg;
    for (int b = j->first; b < j->last; b++) {
        size_t off = (size_t)b * 3 * (size_t)j->n;
        j->energy[b] = sqo_total(j->n, j->L[b], j->xya + off,
                                 j->grad ? j->grad + off : NULL,
                                 j->cand ? j->cand + b : NULL);
    }
    return NULL;
}

/* Energy (+ gradient) of `configs` independent configurations of n squares,
 * threaded over configurations.  Returns the number of threads used. */
int sqo_total_batch(int configs, int n, const double* xya, const double* L,
                    double* energy, double* grad, int64_t* cand, int threads) {
    if (threads < 1) threads = 1;
    if (threads > configs) threads = configs > 0 ? configs : 1;
    pthread_t tid[256];
    sqo_job jobs[256];
    if (threads > 256) threads = 256;
    for (int t = 0; t < threads; t++) {
        jobs[t].first = (int)((int64_t)configs * t / threads);
        jobs[t].last = (int)((int64_t)configs * (t + 1) / threads);
        jobs[t].n = n;
        jobs[t].xya = xya;
        jobs[t].L = L;
        jobs[t].energy = energy;
        jobs[t].grad = grad;
        jobs[t].cand = cand;
        if (t > 0) pthread_create(&tid[t], NULL, sqo_worker, &jobs[t]);
    }
    sqo_worker(&jobs[0]);
    for (int t = 1; t < threads; t++) pthread_join(tid[t], NULL);
    return threads;
}
