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
