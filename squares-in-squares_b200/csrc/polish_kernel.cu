// FP64 gradient polish of every job's best state, one CTA per job.
//
// The reference polishes every chain after every epoch with PRP+ conjugate
// gradient and a 5-step backtracking search on the squared-penetration
// energy at the chain's target side (seeded.cu:621-713, gradient
// pair_cached_smooth :67-90 and the smooth wall derivative :640-645).  Here
// the polish runs once per job on its best FP64 state: compress the state by
// a factor (1 - delta) into a side L (1 - delta), descend the same energy
// with a backtracking line search until it vanishes, and keep the result if
// its dilation-certified side (device_certified_side, seeded.cu:175-226) is
// smaller; delta shrinks after every failure.  Pairs are evaluated all
// against all (n <= 1000, one CTA): every thread owns squares and loops over
// all partners, so gradients need no atomics and reductions have a fixed
// order (the result is deterministic).
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>

#include "anneal.cuh"
#include "common.cuh"

namespace sqs {
namespace ann {

constexpr int kPT = 256;  // threads per polish CTA

// Neighbour lists of the polish: every partner within sqrt(2.000001) + 0.25
// of a square when the list was built (at most kNbK, ascending), valid while
// no square has moved more than 0.125 since -- then every pair inside the
// pair cut-off is listed.  Energies over the list sum the same nonzero terms
// in the same order as the all-pairs loop, so they are bit-identical to it.
constexpr int kNbK = 24;
constexpr double kNbR2 = 2.7697;       // (sqrt(2.000001) + 0.25)^2 = 2.76961, rounded up
constexpr double kNbMove2 = 0.015625;  // 0.125^2

// q0, q, g, sv (double3), cs (double2), the list's reference centres
// (double2), partner indices (uint16) and counts (uint8)
size_t polish_smem_bytes(int n) { return (size_t)n * (4 * 24 + 16 + 16 + 2 * kNbK + 1) + 64; }

__device__ __forceinline__ double sgn_s(double x) { return fabs(x) > 1e-6 ? (x >= 0.0 ? 1.0 : -1.0) : 0.0; }

// Smooth-variant pair gradient for square p against q (pair_cached_smooth):
// returns gap^2 and adds d/dp into g.
__device__ __forceinline__ double pair_smooth(double px, double py, double c, double s, double qx, double qy,
                                              double d, double t, double& gx, double& gy, double& ga) {
    const double dx = qx - px, dy = qy - py;
    if (dx * dx + dy * dy >= 2.000001) return 0.0;
    const double cd = c * d + s * t, sd = s * d - c * t;
    const double rad = 0.5 + 0.5 * (fabs(cd) + fabs(sd));
    const double deriv = 0.5 * (-sgn_s(cd) * sd + sgn_s(sd) * cd);
    const double ux[4] = {c, -s, d, -t}, uy[4] = {s, c, t, d};
    double gap = -1e100, ggx = 0, ggy = 0, gga = 0;
    for (int k = 0; k < 4; ++k) {
        const double v = dx * ux[k] + dy * uy[k], z = fabs(v) - rad;
        if (z > gap) {
            gap = z;
            const double sv = v >= 0.0 ? 1.0 : -1.0;
            ggx = -sv * ux[k];
            ggy = -sv * uy[k];
            gga = -deriv + (k < 2 ? sv * (-dx * uy[k] + dy * ux[k]) : 0.0);
        }
    }
    if (gap >= 0.0) return 0.0;
    gx += 2.0 * gap * ggx;
    gy += 2.0 * gap * ggy;
    ga += 2.0 * gap * gga;
    return gap * gap;
}

__device__ __forceinline__ double wall_smooth(double x, double y, double c, double s, double L, double& gx,
                                              double& gy, double& ga) {
    const double r = 0.5 * (fabs(c) + fabs(s));
    const double dr = 0.5 * (-sgn_s(c) * s + sgn_s(s) * c);
    const double v[4] = {r - x, x + r - L, r - y, y + r - L};
    double e = 0.0;
    for (int k = 0; k < 4; ++k) {
        if (v[k] > 0.0) {
            e += v[k] * v[k];
            const double f = 2.0 * v[k];
            gx += f * (k == 0 ? -1.0 : k == 1 ? 1.0 : 0.0);
            gy += f * (k == 2 ? -1.0 : k == 3 ? 1.0 : 0.0);
            ga += f * dr;
        }
    }
    return e;
}

__device__ double block_sum(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    for (int w = 0; w < kPT / 32; ++w) t += red[w];
    return t;
}

__device__ double block_max(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = red[0];
    for (int w = 1; w < kPT / 32; ++w) t = fmax(t, red[w]);
    return t;
}

struct NbrList {
    double2* ref;   // centres at the build
    uint16_t* idx;  // partners of square i: idx[i * kNbK + k], k < cnt[i]
    uint8_t* cnt;
};

// Energy (and gradient into g when g != nullptr) of the state q at side L,
// over the neighbour list when nb != nullptr, else over all pairs.
__device__ double energy(int n, const double3* q, const double2* cs, double L, double3* g, double* red,
                         const NbrList* nb = nullptr) {
    double e = 0.0;
    for (int i = threadIdx.x; i < n; i += kPT) {
        const double3 p = q[i];
        const double2 pc = cs[i];
        double gx = 0, gy = 0, ga = 0;
        e += wall_smooth(p.x, p.y, pc.x, pc.y, L, gx, gy, ga);
        const int m = nb ? nb->cnt[i] : n;
        for (int k = 0; k < m; ++k) {
            const int j = nb ? (int)nb->idx[i * kNbK + k] : k;
            if (j == i) continue;
            const double3 o = q[j];
            const double2 oc = cs[j];
            double hx = 0, hy = 0, ha = 0;
            const double pe = pair_smooth(p.x, p.y, pc.x, pc.y, o.x, o.y, oc.x, oc.y, hx, hy, ha);
            if (j > i) e += pe;
            gx += hx;
            gy += hy;
            ga += ha;
        }
        if (g) g[i] = make_double3(gx, gy, ga);
    }
    return block_sum(e, red);
}

// Build the list for state q; false when a square has more than kNbK
// partners (the callers then use all pairs).
__device__ bool build_nbr(int n, const NbrList& nb, const double3* q, double* red) {
    double over = 0.0;
    for (int i = threadIdx.x; i < n; i += kPT) {
        const double3 p = q[i];
        int c = 0;
        for (int j = 0; j < n; ++j) {
            if (j == i) continue;
            const double dx = q[j].x - p.x, dy = q[j].y - p.y;
            if (dx * dx + dy * dy < kNbR2) {
                if (c < kNbK) nb.idx[i * kNbK + c] = (uint16_t)j;
                ++c;
            }
        }
        nb.cnt[i] = (uint8_t)min(c, kNbK);
        nb.ref[i] = make_double2(p.x, p.y);
        if (c > kNbK) over = 1.0;
    }
    return block_max(over, red) == 0.0;
}

// Largest squared centre displacement of q since the list was built.
__device__ double moved2(int n, const NbrList& nb, const double3* q, double* red) {
    double m = 0.0;
    for (int i = threadIdx.x; i < n; i += kPT) {
        const double dx = q[i].x - nb.ref[i].x, dy = q[i].y - nb.ref[i].y;
        m = fmax(m, dx * dx + dy * dy);
    }
    return block_max(m, red);
}

// Certified side of q (dilation lambda, bounding box of the dilated state).
__device__ double cert_side_all(int n, const double3* q, const double2* cs, double* red, double& lam_out,
                                double& x0, double& y0) {
    double lam = 1.0;
    for (int i = threadIdx.x; i < n; i += kPT) {
        const double3 p = q[i];
        const double ci = cs[i].x, si = cs[i].y;
        for (int j = i + 1; j < n; ++j) {
            const double dx = p.x - q[j].x, dy = p.y - q[j].y;
            if (dx * dx + dy * dy >= 2.05) continue;
            const double cj = cs[j].x, sj = cs[j].y;
            const double c12 = fabs(ci * cj + si * sj), s12 = fabs(-si * cj + ci * sj);
            const double r = 0.5 + 0.5 * (c12 + s12);
            const double v = fmax(fmax(fabs(dx * ci + dy * si), fabs(-dx * si + dy * ci)),
                                  fmax(fabs(dx * cj + dy * sj), fabs(-dx * sj + dy * cj)));
            lam = fmax(lam, v > 1e-12 ? (r + 2.6e-8) / v : 1e9);
        }
    }
    lam = block_max(lam, red);
    lam_out = lam;
    if (lam > 1.008) return 1e30;
    double a0 = 1e300, a1 = -1e300, b0 = 1e300, b1 = -1e300;
    for (int i = threadIdx.x; i < n; i += kPT) {
        const double r = 0.5 * (fabs(cs[i].x) + fabs(cs[i].y));
        const double x = q[i].x * lam, y = q[i].y * lam;
        a0 = fmin(a0, x - r);
        a1 = fmax(a1, x + r);
        b0 = fmin(b0, y - r);
        b1 = fmax(b1, y + r);
    }
    x0 = -block_max(-a0, red);
    const double xm = block_max(a1, red);
    y0 = -block_max(-b0, red);
    const double ym = block_max(b1, red);
    return fmax(xm - x0, ym - y0);
}

__device__ __forceinline__ double wrap_q(double a) {
    a = fmod(a, 1.57079632679489661923);
    return a < 0.0 ? a + 1.57079632679489661923 : a;
}

__device__ void trig_of(int n, const double3* q, double2* cs) {
    for (int i = threadIdx.x; i < n; i += kPT) {
        double s, c;
        sincos(q[i].z, &s, &c);
        cs[i] = make_double2(c, s);
    }
    __syncthreads();
}

// Shared-memory views of one polish CTA.
struct PolishBufs {
    double3* q0;  // accepted state of the descent
    double3* q;   // trial state
    double3* g;   // gradient at q0
    double3* sv;  // best so far (translated, dilated)
    double2* cs;  // cos/sin of the state being evaluated
    NbrList nb;   // neighbour list of the descent
};

__device__ __forceinline__ PolishBufs polish_bufs(unsigned char* dyn, int n) {
    PolishBufs b;
    b.q0 = reinterpret_cast<double3*>(dyn);
    b.q = b.q0 + n;
    b.g = b.q + n;
    b.sv = b.g + n;
    b.cs = reinterpret_cast<double2*>(b.sv + n);
    b.nb.ref = b.cs + n;
    b.nb.idx = reinterpret_cast<uint16_t*>(b.nb.ref + n);
    b.nb.cnt = reinterpret_cast<uint8_t*>(b.nb.idx + (size_t)n * kNbK);
    return b;
}

// Descend the energy of state q0 at side Lt until it vanishes (at most
// *budget gradient steps, each with up to 8 backtracking trials).
__device__ void descend(int n, const PolishBufs& B, double Lt, int* budget, double* red) {
    trig_of(n, B.q0, B.cs);
    bool listed = build_nbr(n, B.nb, B.q0, red);
    double E = energy(n, B.q0, B.cs, Lt, B.g, red, listed ? &B.nb : nullptr);
    double alpha = 0.05;
    while (*budget > 0 && E > 1e-26) {
        --*budget;
        bool moved = false;
        for (int ls = 0; ls < 8 && !moved; ++ls) {
            for (int i = threadIdx.x; i < n; i += kPT) {
                const double3 p = B.q0[i], d = B.g[i];
                B.q[i] = make_double3(p.x - alpha * d.x, p.y - alpha * d.y, wrap_q(p.z - alpha * d.z));
            }
            __syncthreads();
            trig_of(n, B.q, B.cs);
            const double d2 = listed ? moved2(n, B.nb, B.q, red) : 1e30;
            const double En = energy(n, B.q, B.cs, Lt, nullptr, red, d2 <= kNbMove2 ? &B.nb : nullptr);
            if (En < E) {
                E = En;
                moved = true;
                alpha = fmin(alpha * 1.5, 0.5);
                for (int i = threadIdx.x; i < n; i += kPT) B.q0[i] = B.q[i];
                __syncthreads();
                // keep room for the next trials: rebuild once half the slack is used
                if (d2 > 0.25 * kNbMove2) listed = build_nbr(n, B.nb, B.q0, red);
            } else {
                alpha *= 0.3;
            }
        }
        if (!moved) break;
        E = energy(n, B.q0, B.cs, Lt, B.g, red, listed ? &B.nb : nullptr);  // cs holds the trig of q == q0
    }
    trig_of(n, B.q0, B.cs);
}

// Compress-and-descend attempts on the certified state sv of side *Lb
// (delta shrinking by 0.3 after every attempt that does not certify a
// smaller side); sv and *Lb are updated in place.
__device__ void polish_loop(int n, const PolishBufs& B, double* Lb, int* budget, double* red) {
    double delta = 1e-4;
    for (int attempt = 0; attempt < 12 && *budget > 0 && delta > 1e-9; ++attempt) {
        const double f = 1.0 - delta, Lt = *Lb * f;
        for (int i = threadIdx.x; i < n; i += kPT) B.q0[i] = make_double3(B.sv[i].x * f, B.sv[i].y * f, B.sv[i].z);
        __syncthreads();
        descend(n, B, Lt, budget, red);
        double lam = 0, x0 = 0, y0 = 0;
        const double Lc = cert_side_all(n, B.q0, B.cs, red, lam, x0, y0);
        if (Lc < *Lb) {
            *Lb = Lc;
            for (int i = threadIdx.x; i < n; i += kPT)
                B.sv[i] = make_double3(B.q0[i].x * lam - x0, B.q0[i].y * lam - y0, B.q0[i].z);
            __syncthreads();
        } else {
            delta *= 0.3;
        }
    }
}

__global__ void __launch_bounds__(kPT) polish_kernel(const int32_t* __restrict__ job_list,
                                                     const JobDev* __restrict__ jdev, JobMut* __restrict__ jmut,
                                                     double* __restrict__ best) {
    extern __shared__ __align__(16) unsigned char dyn[];
    __shared__ double red[kPT / 32];
    const int job = job_list[blockIdx.x];
    const JobDev jd = jdev[job];
    const int n = jd.n;
    double Lb = jmut[job].best_L;
    if (jd.polish_iters <= 0 || Lb >= 1e29 || jmut[job].status < 0) return;
    const PolishBufs B = polish_bufs(dyn, n);
    double* b = best + jd.best_off;
    for (int i = threadIdx.x; i < n; i += kPT) B.sv[i] = make_double3(b[3 * i], b[3 * i + 1], b[3 * i + 2]);
    __syncthreads();
    int budget = jd.polish_iters;
    polish_loop(n, B, &Lb, &budget, red);
    for (int i = threadIdx.x; i < n; i += kPT) {
        b[3 * i] = B.sv[i].x;
        b[3 * i + 1] = B.sv[i].y;
        b[3 * i + 2] = B.sv[i].z;
    }
    if (threadIdx.x == 0) jmut[job].best_L = Lb;
}

// Standalone polish of arbitrary states (state k: n_of[k] rows at
// xya + 3 * row0[k], polished in place).  The input's dilation-certified
// side is the incumbent; an input too overlapped to certify (dilation above
// 1.008) first descends its energy inside its own bounding box and, if
// overlaps remain, has its centres spread by that dilation (at most 1.5x)
// and descends in a box scaled alike.
// res[k] = {L_in, L_out, iterations used}.
__global__ void __launch_bounds__(kPT) polish_states_kernel(const int32_t* __restrict__ n_of,
                                                            const int64_t* __restrict__ row0, int iters,
                                                            double* __restrict__ xya, double* __restrict__ res) {
    extern __shared__ __align__(16) unsigned char dyn[];
    __shared__ double red[kPT / 32];
    const int k = blockIdx.x;
    const int n = n_of[k];
    double* st = xya + 3 * row0[k];
    const PolishBufs B = polish_bufs(dyn, n);
    for (int i = threadIdx.x; i < n; i += kPT) B.q0[i] = make_double3(st[3 * i], st[3 * i + 1], wrap_q(st[3 * i + 2]));
    __syncthreads();
    trig_of(n, B.q0, B.cs);
    int budget = iters;
    double lam = 0, x0 = 0, y0 = 0;
    double Lb = cert_side_all(n, B.q0, B.cs, red, lam, x0, y0);
    const double L_in = Lb, lam_in = lam;
    if (Lb >= 1e29) {
        // bounding box of the input, translated to the origin, as the side
        double a0 = 1e300, a1 = -1e300, b0 = 1e300, b1 = -1e300;
        for (int i = threadIdx.x; i < n; i += kPT) {
            const double r = 0.5 * (fabs(B.cs[i].x) + fabs(B.cs[i].y));
            a0 = fmin(a0, B.q0[i].x - r);
            a1 = fmax(a1, B.q0[i].x + r);
            b0 = fmin(b0, B.q0[i].y - r);
            b1 = fmax(b1, B.q0[i].y + r);
        }
        a0 = -block_max(-a0, red);
        a1 = block_max(a1, red);
        b0 = -block_max(-b0, red);
        b1 = block_max(b1, red);
        const double side = fmax(a1 - a0, b1 - b0);
        for (int i = threadIdx.x; i < n; i += kPT) {
            B.sv[i] = make_double3(B.q0[i].x - a0, B.q0[i].y - b0, B.q0[i].z);  // the input, at the origin
            B.q0[i] = B.sv[i];
        }
        __syncthreads();
        // first remove the overlaps inside the input's own bounding box (half
        // the budget); where they do not vanish there, spread the input's
        // centres by the dilation that would separate its close pairs (at
        // most 1.5x) and descend in a box scaled alike
        int half = budget / 2;
        budget -= half;
        descend(n, B, side, &half, red);
        budget += half;
        Lb = cert_side_all(n, B.q0, B.cs, red, lam, x0, y0);
        if (Lb >= 1e29) {
            const double f = fmin(fmax(lam_in, 1.0), 1.5);
            for (int i = threadIdx.x; i < n; i += kPT)
                B.q0[i] = make_double3(B.sv[i].x * f, B.sv[i].y * f, B.sv[i].z);
            __syncthreads();
            descend(n, B, side * f, &budget, red);
            Lb = cert_side_all(n, B.q0, B.cs, red, lam, x0, y0);
        }
    }
    if (Lb < 1e29) {
        for (int i = threadIdx.x; i < n; i += kPT)
            B.sv[i] = make_double3(B.q0[i].x * lam - x0, B.q0[i].y * lam - y0, B.q0[i].z);
        __syncthreads();
        polish_loop(n, B, &Lb, &budget, red);
        for (int i = threadIdx.x; i < n; i += kPT) {
            st[3 * i] = B.sv[i].x;
            st[3 * i + 1] = B.sv[i].y;
            st[3 * i + 2] = B.sv[i].z;
        }
    }
    if (threadIdx.x == 0) {
        res[3 * k] = L_in;
        res[3 * k + 1] = Lb;
        res[3 * k + 2] = (double)(iters - budget);
    }
}

// FP64 energy and gradient of arbitrary states, one CTA per state: the
// polish's own energy function over all pairs (pair_smooth / wall_smooth
// above), with cos and sin taken of the angles as given.  State k has n_of[k]
// rows at xya + 3 * row0[k] and side side[k]; energy[k], and the gradient rows
// at the same offsets of grad when grad is not null.
__global__ void __launch_bounds__(kPT) energy_states_kernel(const int32_t* __restrict__ n_of,
                                                            const int64_t* __restrict__ row0,
                                                            const double* __restrict__ side,
                                                            const double* __restrict__ xya,
                                                            double* __restrict__ energy_out,
                                                            double* __restrict__ grad) {
    extern __shared__ __align__(16) unsigned char dyn[];
    __shared__ double red[kPT / 32];
    const int k = blockIdx.x;
    const int n = n_of[k];
    double3* q = reinterpret_cast<double3*>(dyn);
    double3* g = q + n;
    double2* cs = reinterpret_cast<double2*>(g + n);
    const double* st = xya + 3 * row0[k];
    for (int i = threadIdx.x; i < n; i += kPT) q[i] = make_double3(st[3 * i], st[3 * i + 1], st[3 * i + 2]);
    __syncthreads();
    trig_of(n, q, cs);
    const double e = energy(n, q, cs, side[k], grad ? g : nullptr, red, nullptr);
    if (threadIdx.x == 0) energy_out[k] = e;
    if (grad) {
        double* go = grad + 3 * row0[k];
        for (int i = threadIdx.x; i < n; i += kPT) {
            go[3 * i] = g[i].x;
            go[3 * i + 1] = g[i].y;
            go[3 * i + 2] = g[i].z;
        }
    }
}

size_t energy_smem_bytes(int n) { return (size_t)n * (2 * sizeof(double3) + sizeof(double2)) + 64; }

int launch_energy_states(cudaStream_t stream, int count, const int32_t* n_of, const int64_t* row0, const double* side,
                         const double* xya, double* energy_out, double* grad, size_t smem) {
    static std::atomic<bool> attr_done[64];  // set-up once per device (idempotent if repeated)
    int dev = 0;
    SQS_CUDA(cudaGetDevice(&dev));
    if (!attr_done[dev & 63]) {
        SQS_CUDA(cudaFuncSetAttribute(energy_states_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        attr_done[dev & 63] = true;
    }
    if (count <= 0) return SQS_OK;
    energy_states_kernel<<<count, kPT, smem, stream>>>(n_of, row0, side, xya, energy_out, grad);
    SQS_CUDA(cudaGetLastError());
    return SQS_OK;
}

int launch_polish_states(cudaStream_t stream, int count, const int32_t* n_of, const int64_t* row0, int iters,
                         double* xya, double* res, size_t smem) {
    static std::atomic<bool> attr_done[64];  // set-up once per device (idempotent if repeated)
    int dev = 0;
    SQS_CUDA(cudaGetDevice(&dev));
    if (!attr_done[dev & 63]) {
        SQS_CUDA(cudaFuncSetAttribute(polish_states_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        attr_done[dev & 63] = true;
    }
    if (count <= 0) return SQS_OK;
    polish_states_kernel<<<count, kPT, smem, stream>>>(n_of, row0, iters, xya, res);
    SQS_CUDA(cudaGetLastError());
    return SQS_OK;
}

int launch_polish(cudaStream_t stream, int njobs, const int32_t* job_list, const JobDev* jdev, JobMut* jmut,
                  double* best, size_t smem) {
    static std::atomic<bool> attr_done[64];  // set-up once per device (idempotent if repeated)
    int dev = 0;
    cudaGetDevice(&dev);
    if (!attr_done[dev & 63]) {
        SQS_CUDA(cudaFuncSetAttribute(polish_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        attr_done[dev & 63] = true;
    }
    if (njobs <= 0) return SQS_OK;
    polish_kernel<<<njobs, kPT, smem, stream>>>(job_list, jdev, jmut, best);
    SQS_CUDA(cudaGetLastError());
    return SQS_OK;
}

}  // namespace ann
}  // namespace sqs
