// FP32 cell-list SAT overlap + wall energy and gradient of many independent
// configurations: one CTA per configuration.
//
// Per CTA (all in shared memory):
//   1. load the n squares (coalesced 12-byte records), cos/sin, wall term,
//      cell id on a G x G grid of cells with side >= sqrt(2.000001) (so every
//      interacting pair sits in the same or adjacent cells), per-cell counts;
//   2. exclusive scan of the counts, counting-sort scatter, each cell's few
//      entries ordered by square index (deterministic pair order);
//   3. broad phase: every square scans two contiguous ranges of the
//      cell-sorted array -- the rest of its own cell plus the east cell, and
//      the three cells of the row above -- which visits each unordered
//      neighbour pair exactly once.  Pairs inside the cut-off are appended
//      to a per-warp queue (ballot + popc), and every time 32 are queued the
//      whole warp evaluates them (narrow phase at full SIMT width), adding
//      both squares' gradients with shared-memory atomics;
//   4. warp-shuffle + shared reduction of the energy and candidate count,
//      coalesced store of the gradient.
// Reference: total_cached (seeded.cu:148-162) is the all-pairs O(n^2) form
// of the same energy; the legacy FP32 path's 16x16 cell grid of width 2
// (packing.cu:22-47) is the reference's own cell-list idea.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "sat_pair.cuh"

namespace sqs {

constexpr int kSatMaxN = 1024;
constexpr float kCellMin = 1.41422f;  // > sqrt(2.000001) = 1.4142139
constexpr int kQueue = 64;            // per-warp pair queue entries

// Gradient accumulation with native 32-bit integer shared-memory atomics
// (shared-memory float atomics are several times slower): a contribution v
// is split into floor(v * 2^12) and the remaining fraction in units of 2^-32,
// two integer sums that cannot overflow for n <= 1024 (|v| < 6 per pair) and
// that do not depend on the order of the additions.
struct GradFix {
    int* hi;        // [3n]
    unsigned* lo;   // [3n]
    __device__ __forceinline__ void add(int k, float v) const {
        const float s = v * 4096.0f;
        const float f = floorf(s);
        atomicAdd(hi + k, (int)f);
        atomicAdd(lo + k, __float2uint_rn((s - f) * 1048576.0f));
    }
    __device__ __forceinline__ float value(int k) const {
        return (float)(((double)hi[k] + (double)lo[k] * (1.0 / 1048576.0)) * (1.0 / 4096.0));
    }
};

__host__ __device__ inline int sat_grid_cap(int n) {
    // Cell grid side cap: about sqrt(2n) cells per side, at most 45 (L = 64).
    int g = (int)sqrtf(2.0f * (float)n);
    return g < 1 ? 1 : (g > 45 ? 45 : g);
}

__host__ __device__ inline size_t sat_smem_bytes(int n, int threads) {
    const int G = sat_grid_cap(n);
    size_t b = 0;
    b += (size_t)n * 16;                      // stash (x, y, c, s) by original index
    b += (size_t)n * 16;                      // cell-sorted (x, y) and (c, s)
    b += (size_t)n * 12;                      // wall gradient by original index
    b += (size_t)n * 24;                      // pair gradient accumulators (GradFix)
    b += (size_t)n * 4;                       // sorted -> (original index, cell)
    b += (size_t)n * 4;                       // original -> (cell, rank)
    b += (size_t)(G * G + 1) * 4;             // cell counts / starts
    b += (size_t)(threads / 32) * kQueue * 4; // warp pair queues
    b += 64;                                  // reduction scratch
    return (b + 15) & ~(size_t)15;
}

template <int T>
__global__ void __launch_bounds__(T) sat_energy_kernel(int n, const float* __restrict__ xya,
                                                        const float* __restrict__ side,
                                                        float* __restrict__ energy,
                                                        float* __restrict__ grad,
                                                        uint32_t* __restrict__ cand) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int W = T / 32;
    const int cfg = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int Gcap = sat_grid_cap(n);
    float4* stash = reinterpret_cast<float4*>(smem);
    float2* sxy = reinterpret_cast<float2*>(stash + n);             // cell-sorted centres
    float2* scs = sxy + n;                                          // cell-sorted cos/sin
    float* gacc = reinterpret_cast<float*>(scs + n);                // wall gradient
    GradFix gf{reinterpret_cast<int*>(gacc + 3 * n), reinterpret_cast<unsigned*>(gacc + 6 * n)};
    short2* sorted_meta = reinterpret_cast<short2*>(gacc + 9 * n);  // (orig, cell)
    short2* orig_meta = sorted_meta + n;                            // (cell, rank)
    int* cells = reinterpret_cast<int*>(orig_meta + n);             // G*G + 1
    uint32_t* queues = reinterpret_cast<uint32_t*>(cells + Gcap * Gcap + 1);
    float* red = reinterpret_cast<float*>(queues + W * kQueue);

    const float L = side[cfg];
    int G = (int)(L / kCellMin);
    G = G < 1 ? 1 : (G > Gcap ? Gcap : G);
    const float inv_cell = (float)G / L;
    const int ncell = G * G;

    for (int c = tid; c <= ncell; c += T) cells[c] = 0;
    __syncthreads();

    // 1. load, trig, walls, cell binning
    float e_loc = 0.f;
    const float* src = xya + (size_t)cfg * 3 * n;
    for (int i = tid; i < n; i += T) {
        const float x = src[3 * i], y = src[3 * i + 1], a = src[3 * i + 2];
        float s, c;
        sincosf(a, &s, &c);
        float gx = 0.f, gy = 0.f, ga = 0.f;
        e_loc += wall_energy_grad(x, y, c, s, L, gx, gy, ga);
        gacc[3 * i] = gx;
        gacc[3 * i + 1] = gy;
        gacc[3 * i + 2] = ga;
        int cx = (int)floorf(x * inv_cell), cy = (int)floorf(y * inv_cell);
        cx = cx < 0 ? 0 : (cx >= G ? G - 1 : cx);
        cy = cy < 0 ? 0 : (cy >= G ? G - 1 : cy);
        const int cell = cy * G + cx;
        const int rank = atomicAdd(&cells[cell], 1);
        stash[i] = make_float4(x, y, c, s);
        orig_meta[i] = make_short2((short)cell, (short)rank);
    }
    __syncthreads();

    // 2. exclusive scan over ncell counts (one warp; ncell <= 2025)
    if (tid < 32) {
        const int per = (ncell + 31) / 32;
        const int lo = tid * per, hi = min(lo + per, ncell);
        int sum = 0;
        for (int c = lo; c < hi; ++c) sum += cells[c];
        int incl = sum;
        for (int o = 1; o < 32; o <<= 1) {
            int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (tid >= o) incl += v;
        }
        int run = incl - sum;
        for (int c = lo; c < hi; ++c) {
            int k = cells[c];
            cells[c] = run;
            run += k;
        }
        if (tid == 31) cells[ncell] = incl;
    }
    __syncthreads();
    for (int i = tid; i < n; i += T) {
        const short2 m = orig_meta[i];
        const int pos = cells[m.x] + m.y;
        const float4 v = stash[i];
        sxy[pos] = make_float2(v.x, v.y);
        scs[pos] = make_float2(v.z, v.w);
        sorted_meta[pos] = make_short2((short)i, m.x);
    }
    __syncthreads();
    // order each cell's entries by original index (cells hold a few squares)
    for (int c = tid; c < ncell; c += T) {
        const int a = cells[c], b = cells[c + 1];
        for (int u = a + 1; u < b; ++u) {
            const float2 kxy = sxy[u], kcs = scs[u];
            const short2 km = sorted_meta[u];
            int w = u - 1;
            while (w >= a && sorted_meta[w].x > km.x) {
                sxy[w + 1] = sxy[w];
                scs[w + 1] = scs[w];
                sorted_meta[w + 1] = sorted_meta[w];
                --w;
            }
            sxy[w + 1] = kxy;
            scs[w + 1] = kcs;
            sorted_meta[w + 1] = km;
        }
    }
    for (int k = tid; k < 3 * n; k += T) {
        gf.hi[k] = 0;
        gf.lo[k] = 0u;
    }
    __syncthreads();

    // 3. broad phase into warp queues, narrow phase 32 pairs at a time
    uint32_t cand_loc = 0;
    uint32_t* queue = queues + warp * kQueue;
    int qn = 0;  // warp-uniform queue length
    auto narrow = [&](uint32_t entry) {
        const int p = (int)(entry & 0xffffu), q = (int)(entry >> 16);
        const float2 P = sxy[p], Q = sxy[q], Pc = scs[p], Qc = scs[q];
        PairGrad g;
        if (sat_pair_grad(Q.x - P.x, Q.y - P.y, Pc.x, Pc.y, Qc.x, Qc.y, g)) {
            e_loc += g.e;
            const int i = sorted_meta[p].x, j = sorted_meta[q].x;
            gf.add(3 * i, g.px);
            gf.add(3 * i + 1, g.py);
            gf.add(3 * i + 2, g.pa);
            gf.add(3 * j, g.qx);
            gf.add(3 * j + 1, g.qy);
            gf.add(3 * j + 2, g.qa);
        }
    };
    for (int base = warp * 32; base < n; base += T) {
        const int p = base + lane;
        int a1 = 0, len1 = 0, a2 = 0, len = 0;
        float px = 0.f, py = 0.f;
        if (p < n) {
            const float2 P = sxy[p];
            px = P.x;
            py = P.y;
            const int cell = sorted_meta[p].y, cy = cell / G, cx = cell - cy * G;
            // own cell after p, then the east cell (same row, contiguous)
            a1 = p + 1;
            len1 = cells[cy * G + min(cx + 2, G)] - a1;
            // the row above: cells cx-1 .. cx+1
            int len2 = 0;
            if (cy + 1 < G) {
                a2 = cells[(cy + 1) * G + max(cx - 1, 0)];
                len2 = cells[(cy + 1) * G + min(cx + 2, G)] - a2;
            }
            len = len1 + len2;
        }
        const int maxlen = __reduce_max_sync(0xffffffffu, len);
        for (int t = 0; t < maxlen; ++t) {
            bool pass = false;
            int q = 0;
            if (t < len) {
                q = t < len1 ? a1 + t : a2 + (t - len1);
                const float2 Q = sxy[q];
                const float dx = Q.x - px, dy = Q.y - py;
                const float d2 = dx * dx + dy * dy;
                pass = d2 < kPairCut2;
                cand_loc += d2 < 2.0f;
            }
            const uint32_t m = __ballot_sync(0xffffffffu, pass);
            if (pass) queue[qn + __popc(m & ((1u << lane) - 1u))] = (uint32_t)p | ((uint32_t)q << 16);
            qn += __popc(m);
            if (qn >= 32) {
                __syncwarp();
                narrow(queue[lane]);
                __syncwarp();
                if (lane < qn - 32) queue[lane] = queue[32 + lane];
                __syncwarp();
                qn -= 32;
            }
        }
    }
    __syncwarp();
    if (lane < qn) narrow(queue[lane]);
    __syncthreads();

    // 4. reductions and stores
    for (int o = 16; o > 0; o >>= 1) {
        e_loc += __shfl_xor_sync(0xffffffffu, e_loc, o);
        cand_loc += __shfl_xor_sync(0xffffffffu, cand_loc, o);
    }
    if (lane == 0) {
        red[warp] = e_loc;
        reinterpret_cast<uint32_t*>(red)[W + warp] = cand_loc;
    }
    __syncthreads();
    if (tid == 0) {
        float e = 0.f;
        uint32_t cc = 0;
        for (int w = 0; w < W; ++w) {
            e += red[w];
            cc += reinterpret_cast<uint32_t*>(red)[W + w];
        }
        energy[cfg] = e;
        if (cand) cand[cfg] = cc;
    }
    if (grad) {
        float* dst = grad + (size_t)cfg * 3 * n;
        for (int k = tid; k < 3 * n; k += T) dst[k] = gacc[k] + gf.value(k);
    }
}

// ---------------------------------------------------------------------------
// Warp-per-configuration form for n <= 256: the same phases as above run by
// one warp without block barriers, several configurations per CTA, except that
// energies are summed exactly as integers, so a cell's entries need no ordering.  A lane
// keeps its (up to 8) squares in registers from the load to the scatter, all
// loads are issued before any is used, and the cell grid is sized from n, so
// ~7.7 KB of shared memory per configuration lets a whole 4,096-configuration
// batch be resident in one wave.
constexpr int kWarpMaxN = 256;
constexpr int kWarpNpl = kWarpMaxN / 32;

__host__ __device__ inline int warp_grid_cap(int n) {
    int g = (int)sqrtf((float)n) + 2;
    return g > 45 ? 45 : g;
}

__host__ __device__ inline size_t warp_smem_bytes(int n) {
    const int G = warp_grid_cap(n);
    // sorted (x, y) + (c, s), pair-gradient accumulators, original index (byte),
    // cell starts (uint16), pair queue
    size_t b = (size_t)n * 16 + (size_t)n * 12 + (((size_t)n + 3) & ~(size_t)3) +
               (((size_t)(G * G + 1) * 2 + 3) & ~(size_t)3) + kQueue * 4;
    return (b + 15) & ~(size_t)15;
}

// Pair-gradient sums of the warp kernel: one 32-bit integer per component in
// units of 2^-19.  A pair term is bounded by 2 r_max (|d| + 1/sqrt 2) =
// 2 * 1.2071 * 2.1213 < 5.13, so with n <= 256 (at most 255 partners) a sum
// stays below 2^31 units; every term is rounded once (error < 1e-6) and the
// sum is exact and order-free.
constexpr float kGScale = 524288.0f;

// Energies of the warp kernel are summed as 64-bit integers in units of
// 2^-40: every wall and pair term is rounded once (error below 5e-13), the
// sum is exact, and so it does not depend on the order in which the pairs are
// found -- cell lists built with atomics need no sorting for a deterministic
// result.  A configuration's energy is far below 2^23, so the sum stays
// below 2^63 units.
constexpr double kEUnit = 1099511627776.0;  // 2^40
__device__ __forceinline__ long long e_units(float e) { return __float2ll_rn(e * 1099511627776.0f); }

// round(v * kGScale) to the nearest integer (ties to even) on the FMA pipe:
// for |v * kGScale| < 2^22 the fused v * 2^19 + 1.5 * 2^23 lands in
// [2^23, 2^24), where one float ulp is 1, so its bit pattern minus that of
// 1.5 * 2^23 is the rounded integer.  |v| < 5.13 keeps it within range.
__device__ __forceinline__ int gq_units(float v) {
    return __float_as_int(fmaf(v, kGScale, 12582912.0f)) - 0x4B400000;
}

// 28 / W CTAs of W warps per SM (72 registers a thread at W = 4; the default
// is W = 2, measured 2% faster than 4 and 20% faster than 8): with the
// shared memory of n = 200 that keeps 4,096 configurations in one wave.
template <int W, bool COUNT>
__global__ void __launch_bounds__(W * 32, 28 / W) sat_energy_warp_kernel(int configs, int n, const float* __restrict__ xya,
                                                                 const float* __restrict__ side,
                                                                 float* __restrict__ energy, float* __restrict__ grad,
                                                                 uint32_t* __restrict__ cand) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int cfg = blockIdx.x * W + warp;
    if (cfg >= configs) return;
    const size_t wb = warp_smem_bytes(n);
    unsigned char* base = smem + (size_t)warp * wb;
    const int Gcap = warp_grid_cap(n);
    float2* sxy = reinterpret_cast<float2*>(base);            // cell-sorted centres
    float2* scs = sxy + n;                                     // cell-sorted cos/sin
    int* gq = reinterpret_cast<int*>(scs + n);                 // pair-gradient sums (kGScale units)
    uint8_t* orig = reinterpret_cast<uint8_t*>(gq + 3 * n);    // sorted -> original index
    uint16_t* cells = reinterpret_cast<uint16_t*>(orig + ((n + 3) & ~3));  // G*G + 1 starts
    uint32_t* queue = reinterpret_cast<uint32_t*>(cells + (((Gcap * Gcap + 1) + 1) & ~1));

    const float L = side[cfg];
    int G = (int)(L / kCellMin);
    G = G < 1 ? 1 : (G > Gcap ? Gcap : G);
    const float inv_cell = (float)G / L;
    const int ncell = G * G;
    for (int c = lane; c <= ncell; c += 32) cells[c] = 0;
    float* gdst = grad ? grad + (size_t)cfg * 3 * n : nullptr;

    // 1. all loads first, then trig, walls and cell ranks
    const float* src = xya + (size_t)cfg * 3 * n;
    float px[kWarpNpl], py[kWarpNpl], pa[kWarpNpl];
#pragma unroll
    for (int k = 0; k < kWarpNpl; ++k) {
        const int i = lane + 32 * k;
        if (i < n) {
            px[k] = src[3 * i];
            py[k] = src[3 * i + 1];
            pa[k] = src[3 * i + 2];
        }
    }
    __syncwarp();
    long long e_loc = 0;  // kEUnit units: exact, so the sum does not depend on the order of the pairs
    float pc[kWarpNpl], ps[kWarpNpl];
    int cr[kWarpNpl];  // cell << 16 | rank
#pragma unroll
    for (int k = 0; k < kWarpNpl; ++k) {
        const int i = lane + 32 * k;
        if (i < n) {
            sincosf(pa[k], &ps[k], &pc[k]);
            float gx = 0.f, gy = 0.f, ga = 0.f;
            e_loc += e_units(wall_energy_grad(px[k], py[k], pc[k], ps[k], L, gx, gy, ga));
            if (gdst) {  // the wall term goes straight out (unbounded for squares far outside
                         // the box); pair terms are added at the end
                gdst[3 * i] = gx;
                gdst[3 * i + 1] = gy;
                gdst[3 * i + 2] = ga;
            }
            gq[3 * i] = gq[3 * i + 1] = gq[3 * i + 2] = 0;
            int cx = (int)floorf(px[k] * inv_cell), cy = (int)floorf(py[k] * inv_cell);
            cx = cx < 0 ? 0 : (cx >= G ? G - 1 : cx);
            cy = cy < 0 ? 0 : (cy >= G ? G - 1 : cy);
            const int cell = cy * G + cx;
            // per-cell counts in 16-bit halves of 32-bit words (native integer atomics)
            const unsigned old = atomicAdd(reinterpret_cast<unsigned*>(cells) + (cell >> 1), 1u << (16 * (cell & 1)));
            cr[k] = (cell << 16) | (int)((old >> (16 * (cell & 1))) & 0xffffu);
        }
    }
    __syncwarp();
    // 2. exclusive scan of the cell counts, scatter from registers
    {
        const int per = (ncell + 31) / 32;
        const int lo = lane * per, hi = min(lo + per, ncell);
        int sum = 0;
        for (int c = lo; c < hi; ++c) sum += cells[c];
        int incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        int run = incl - sum;
        for (int c = lo; c < hi; ++c) {
            const int k = cells[c];
            cells[c] = run;
            run += k;
        }
        if (lane == 31) cells[ncell] = incl;
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < kWarpNpl; ++k) {
        const int i = lane + 32 * k;
        if (i < n) {
            const int cell = cr[k] >> 16;
            const int pos = cells[cell] + (cr[k] & 0xffff);
            sxy[pos] = make_float2(px[k], py[k]);
            scs[pos] = make_float2(pc[k], ps[k]);
            orig[pos] = (uint8_t)i;
        }
    }
    __syncwarp();

    // 3. broad phase into the warp queue, narrow phase 32 pairs at a time
    uint32_t cand_loc = 0;
    int qn = 0;
    auto narrow = [&](uint32_t entry) {
        const int p = (int)(entry & 0xffffu), q = (int)(entry >> 16);
        const float2 P = sxy[p], Q = sxy[q], Pc = scs[p], Qc = scs[q];
        PairGrad g;
        if (sat_pair_grad(Q.x - P.x, Q.y - P.y, Pc.x, Pc.y, Qc.x, Qc.y, g)) {
            e_loc += e_units(g.e);
            const int i = orig[p], j = orig[q];
            atomicAdd(gq + 3 * i, gq_units(g.px));
            atomicAdd(gq + 3 * i + 1, gq_units(g.py));
            atomicAdd(gq + 3 * i + 2, gq_units(g.pa));
            atomicAdd(gq + 3 * j, gq_units(g.qx));
            atomicAdd(gq + 3 * j + 1, gq_units(g.qy));
            atomicAdd(gq + 3 * j + 2, gq_units(g.qa));
        }
    };
    for (int base0 = 0; base0 < n; base0 += 32) {
        const int p = base0 + lane;
        int a1 = 0, len1 = 0, a2 = 0, len = 0;
        float qx0 = 0.f, qy0 = 0.f;
        if (p < n) {
            const float2 P = sxy[p];
            qx0 = P.x;
            qy0 = P.y;
            int cx = (int)floorf(P.x * inv_cell), cy = (int)floorf(P.y * inv_cell);
            cx = cx < 0 ? 0 : (cx >= G ? G - 1 : cx);
            cy = cy < 0 ? 0 : (cy >= G ? G - 1 : cy);
            a1 = p + 1;
            len1 = cells[cy * G + min(cx + 2, G)] - a1;
            int len2 = 0;
            if (cy + 1 < G) {
                a2 = cells[(cy + 1) * G + max(cx - 1, 0)];
                len2 = cells[(cy + 1) * G + min(cx + 2, G)] - a2;
            }
            len = len1 + len2;
            a2 -= len1;  // q = a2 + t for t >= len1
        }
        const int maxlen = __reduce_max_sync(0xffffffffu, len);
        for (int t = 0; t < maxlen; ++t) {
            bool pass = false;
            int q = 0;
            if (t < len) {
                q = (t < len1 ? a1 : a2) + t;
                const float2 Q = sxy[q];
                const float dx = Q.x - qx0, dy = Q.y - qy0;
                const float d2 = dx * dx + dy * dy;
                pass = d2 < kPairCut2;
                if (COUNT) cand_loc += d2 < 2.0f;
            }
            const uint32_t m = __ballot_sync(0xffffffffu, pass);
            if (pass) queue[qn + __popc(m & ((1u << lane) - 1u))] = (uint32_t)p | ((uint32_t)q << 16);
            qn += __popc(m);
            if (qn >= 32) {
                __syncwarp();
                narrow(queue[lane]);
                __syncwarp();
                if (lane < qn - 32) queue[lane] = queue[32 + lane];
                __syncwarp();
                qn -= 32;
            }
        }
    }
    __syncwarp();
    if (lane < qn) narrow(queue[lane]);
    __syncwarp();

    // 4. reductions and the coalesced gradient store
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        e_loc += __shfl_xor_sync(0xffffffffu, e_loc, o);
        cand_loc += __shfl_xor_sync(0xffffffffu, cand_loc, o);
    }
    if (lane == 0) {
        energy[cfg] = (float)((double)e_loc * (1.0 / kEUnit));
        if (COUNT) cand[cfg] = cand_loc;
    }
    if (gdst) {
        for (int k = lane; k < 3 * n; k += 32) gdst[k] += (float)gq[k] * (1.0f / kGScale);
    }
}

template <int W>
static int launch_warp(sqs_ctx* ctx, cudaStream_t st, int configs, int n, const float* xya, const float* side,
                       float* energy, float* grad, uint32_t* cand) {
    const size_t smem = warp_smem_bytes(n) * W;
    static bool attr_set[64] = {false};
    const int dev = ctx->device & 63;
    if (!attr_set[dev]) {
        SQS_CUDA(cudaFuncSetAttribute(sat_energy_warp_kernel<W, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      200 * 1024));
        SQS_CUDA(cudaFuncSetAttribute(sat_energy_warp_kernel<W, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      200 * 1024));
        attr_set[dev] = true;
    }
    const unsigned blocks = (unsigned)((configs + W - 1) / W);
    if (cand)
        sat_energy_warp_kernel<W, true><<<blocks, W * 32, smem, st>>>(configs, n, xya, side, energy, grad,
                                                                               cand);
    else
        sat_energy_warp_kernel<W, false><<<blocks, W * 32, smem, st>>>(configs, n, xya, side, energy, grad,
                                                                                nullptr);
    SQS_CUDA(cudaGetLastError());
    ctx->launches += 1;
    return SQS_OK;
}

template <int T>
static int launch(sqs_ctx* ctx, cudaStream_t st, int configs, int n, const float* xya, const float* side,
                  float* energy, float* grad, uint32_t* cand) {
    const size_t smem = sat_smem_bytes(n, T);
    static bool attr_set[64] = {false};
    const int dev = ctx->device & 63;
    if (!attr_set[dev]) {
        SQS_CUDA(cudaFuncSetAttribute(sat_energy_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      96 * 1024));
        attr_set[dev] = true;
    }
    sat_energy_kernel<T><<<configs, T, smem, st>>>(n, xya, side, energy, grad, cand);
    SQS_CUDA(cudaGetLastError());
    ctx->launches += 1;
    return SQS_OK;
}

static int sat_energy_launch_on(sqs_ctx* ctx, cudaStream_t st, int configs, int n, const float* xya,
                                const float* side, float* energy, float* grad, uint32_t* cand, int threads) {
    SQS_REQUIRE(configs >= 0 && configs <= (1 << 30), "configs %d out of range", configs);
    SQS_REQUIRE(n >= 1 && n <= kSatMaxN, "n %d out of 1..%d", n, kSatMaxN);
    SQS_REQUIRE(xya && side && energy, "null device pointer");
    if (configs == 0) return SQS_OK;
    if (threads == 0) threads = n <= kWarpMaxN ? -2 : 128;
    if (threads < 0) {  // warp-per-configuration kernel, -threads warps per CTA
        SQS_REQUIRE(n <= kWarpMaxN, "the warp-per-configuration kernel takes n <= %d", kWarpMaxN);
        switch (-threads) {
            case 2: return launch_warp<2>(ctx, st, configs, n, xya, side, energy, grad, cand);
            case 4: return launch_warp<4>(ctx, st, configs, n, xya, side, energy, grad, cand);
            case 8: return launch_warp<8>(ctx, st, configs, n, xya, side, energy, grad, cand);
            default: break;
        }
        SQS_REQUIRE(false, "threads %d: warps per CTA must be 2, 4 or 8", threads);
    }
    switch (threads) {
        case 32: return launch<32>(ctx, st, configs, n, xya, side, energy, grad, cand);
        case 64: return launch<64>(ctx, st, configs, n, xya, side, energy, grad, cand);
        case 128: return launch<128>(ctx, st, configs, n, xya, side, energy, grad, cand);
        case 256: return launch<256>(ctx, st, configs, n, xya, side, energy, grad, cand);
        default: break;
    }
    SQS_REQUIRE(false, "threads %d not in {32, 64, 128, 256}", threads);
}

int sat_energy_launch(sqs_ctx* ctx, int configs, int n, const float* xya, const float* side,
                      float* energy, float* grad, uint32_t* cand, int threads) {
    return sat_energy_launch_on(ctx, ctx->stream, configs, n, xya, side, energy, grad, cand, threads);
}

}  // namespace sqs

extern "C" int sqs_sat_energy(sqs_ctx* ctx, int configs, int n, const float* xya, const float* side,
                              float* energy, float* grad, uint32_t* cand, int threads) {
    if (int r = sqs::enter(ctx)) return r;
    return sqs::sat_energy_launch(ctx, configs, n, xya, side, energy, grad, cand, threads);
}

extern "C" int sqs_sat_energy_host(sqs_ctx* ctx, int configs, int n, const float* xya,
                                   const float* side, float* energy, float* grad, uint32_t* cand) {
    if (int r = sqs::enter(ctx)) return r;
    SQS_REQUIRE(configs >= 0 && n >= 1 && n <= sqs::kSatMaxN, "configs/n out of range");
    SQS_REQUIRE(xya && side && energy, "null host pointer");
    if (configs == 0) return SQS_OK;
    const size_t sb = (size_t)configs * n * 3 * sizeof(float);
    if (int r = ctx->d_in.reserve(sb)) return r;
    if (int r = ctx->d_side.reserve((size_t)configs * sizeof(float))) return r;
    if (int r = ctx->d_out.reserve((size_t)configs * sizeof(float))) return r;
    if (grad)
        if (int r = ctx->d_grad.reserve(sb)) return r;
    if (cand)
        if (int r = ctx->d_cand.reserve((size_t)configs * sizeof(uint32_t))) return r;
    // Chunks of the batch on the context's side streams: the upload of one
    // chunk, the kernel of the one before and the download of the one before
    // that overlap.  Four chunks measured best for 4,096 x 200 squares
    // (0.38 ms per call against 0.44 ms in one piece; 8 and 16 chunks cost
    // more in calls than they gain: the host link carried about 51 GB/s in
    // both directions together, so the transfers overlap only in part).
    const int chunks = configs >= 1024 ? std::min(4, configs / 256) : 1;
    float* d_in = (float*)ctx->d_in.p;
    float* d_side = (float*)ctx->d_side.p;
    float* d_out = (float*)ctx->d_out.p;
    float* d_grad = grad ? (float*)ctx->d_grad.p : nullptr;
    uint32_t* d_cand = cand ? (uint32_t*)ctx->d_cand.p : nullptr;
    const int na = chunks == 1 ? 0 : std::min(chunks, sqs_ctx::kAux);
    SQS_CUDA(cudaEventRecord(ctx->fork, ctx->stream));
    for (int a = 0; a < na; ++a) SQS_CUDA(cudaStreamWaitEvent(ctx->aux[a], ctx->fork, 0));
    int rc = SQS_OK;
    for (int c = 0; c < chunks && rc == SQS_OK; ++c) {
        cudaStream_t st = chunks == 1 ? ctx->stream : ctx->aux[c % sqs_ctx::kAux];
        const int64_t lo = (int64_t)configs * c / chunks, hi = (int64_t)configs * (c + 1) / chunks;
        const int cnt = (int)(hi - lo);
        const size_t e0 = (size_t)lo * n * 3, eb = (size_t)cnt * n * 3 * sizeof(float);
        SQS_CUDA(cudaMemcpyAsync(d_in + e0, xya + e0, eb, cudaMemcpyHostToDevice, st));
        SQS_CUDA(cudaMemcpyAsync(d_side + lo, side + lo, (size_t)cnt * sizeof(float), cudaMemcpyHostToDevice, st));
        rc = sqs::sat_energy_launch_on(ctx, st, cnt, n, d_in + e0, d_side + lo, d_out + lo,
                                       d_grad ? d_grad + e0 : nullptr, d_cand ? d_cand + lo : nullptr, 0);
        if (rc) break;
        SQS_CUDA(cudaMemcpyAsync(energy + lo, d_out + lo, (size_t)cnt * sizeof(float), cudaMemcpyDeviceToHost, st));
        if (grad) SQS_CUDA(cudaMemcpyAsync(grad + e0, d_grad + e0, eb, cudaMemcpyDeviceToHost, st));
        if (cand)
            SQS_CUDA(cudaMemcpyAsync(cand + lo, d_cand + lo, (size_t)cnt * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                     st));
    }
    // join every side stream, also after a failure
    for (int a = 0; a < na; ++a) {
        SQS_CUDA(cudaEventRecord(ctx->join[a], ctx->aux[a]));
        SQS_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->join[a], 0));
    }
    if (rc) return rc;
    SQS_CUDA(cudaStreamSynchronize(ctx->stream));
    return SQS_OK;
}
