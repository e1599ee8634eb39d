// Batched parallel-tempering simulated annealing of unit squares in a
// shrinking square container: one thread-block cluster per job, one warp per
// replica, every replica's squares and cell list in shared memory.
//
// Reference semantics it re-designs (cuda/seeded.cu): the energy model
// (pair_cached/boundary/total_cached :41-162), single-square Metropolis
// moves (:501-546), replica exchange within a temperature ladder
// (swap_replicas :791-817), the FP64 dilation-certified side of a candidate
// best state (device_certified_side :175-226) and the host's shrink of the
// container after every improvement (:919-938).  What is new:
//   * FP32 moves and energies, with dE of a single-square move taken over the
//     3x3 cell neighbourhood (O(1) per proposal instead of O(n));
//   * lanes of the replica's warp split the neighbour candidates, a butterfly
//     reduction leaves the same dE on every lane, so every lane takes the same
//     Metropolis decision without a broadcast;
//   * counter-based Philox keyed by (job seed, replica, proposal index): a
//     job's trajectory does not depend on the batch, slot or CTA running it;
//   * replica exchange swaps rungs (temperature indices), not states, and the
//     whole ladder (up to 64 rungs) may span a cluster of CTAs, exchanged over
//     distributed shared memory;
//   * the shrink decision is taken on the device at every exchange point
//     (no per-epoch device-to-host round trip).
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <tuple>
#include <mutex>
#include <map>

#include <cmath>

#include "anneal.cuh"
#include "common.cuh"
#include "philox.cuh"
#include "sat_pair.cuh"

namespace cg = cooperative_groups;

namespace sqs {
namespace ann {

constexpr float kHalfPiF = 1.57079632679489662f;

// cos/sin of a replica's angle, wherever the state's trig is (re)computed:
// CUDA's full-accuracy sincosf, the same function everywhere so a state's
// (cos, sin) never depends on where it was computed (a sliced run reloads what
// an unsliced one kept).  Against the hardware approximation it costs about 3%
// of the proposal rate and cuts the FP32 energies' absolute error against the
// FP64 oracle about eightfold (measured on the batched and served samples), to
// well inside the 1e-5 floor.  The FP64 certified side recomputes trig from
// the angle itself.
__device__ __forceinline__ void state_trig(float a, float* s, float* c) { sincosf(a, s, c); }

struct Rep {  // one replica's shared-memory view
    float4* sq;        // (x, y, cos a, sin a)
    float* ang;        // a in [0, pi/2)
    uint8_t* cnt;      // squares per cell
    uint16_t* slot;    // cell c: slot[c * kCellK + k]
};

__device__ __forceinline__ Rep rep_view(unsigned char* base, int n, int Gmax) {
    Rep r;
    r.sq = reinterpret_cast<float4*>(base);
    r.ang = reinterpret_cast<float*>(r.sq + n);
    r.cnt = reinterpret_cast<uint8_t*>(r.ang + n);
    r.slot = reinterpret_cast<uint16_t*>(r.cnt + ((Gmax * Gmax + 3) & ~3));
    return r;
}

struct Grid {
    int G;
    float inv;  // G / L
    __device__ __forceinline__ int cx(float x) const {
        int c = (int)floorf(x * inv);
        return c < 0 ? 0 : (c >= G ? G - 1 : c);
    }
};

__device__ __forceinline__ Grid make_grid(float L, int Gmax, float cell) {
    Grid g;
    int G = (int)(L / cell);
    g.G = G < 1 ? 1 : (G > Gmax ? Gmax : G);
    g.inv = (float)g.G / L;
    return g;
}

__device__ __forceinline__ float wall_e(float x, float y, float c, float s, float L) {
    return wall_energy(x, y, c, s, L);
}

// Build the cell list of one replica (warp).  Returns false on overflow (a
// cell asked for more than kCellK slots); the list is then incomplete but
// every count is clamped to kCellK and every slot holds a valid index, so no
// later scan can leave the replica's arrays.
__device__ bool build_cells(const Rep& R, int n, const Grid& g, int lane) {
    const int ncell = g.G * g.G;
    for (int c = lane; c < ncell; c += 32) R.cnt[c] = 0;
    for (int k = lane; k < ncell * kCellK; k += 32) R.slot[k] = 0;
    __syncwarp();
    bool ok = true;
    for (int i = lane; i < n; i += 32) {
        const float4 p = R.sq[i];
        const int c = g.cx(p.y) * g.G + g.cx(p.x);
        const unsigned k = atomicAdd(reinterpret_cast<unsigned*>(R.cnt + (c & ~3)), 1u << (8 * (c & 3)));
        const unsigned slot_k = (k >> (8 * (c & 3))) & 0xffu;
        if (slot_k < (unsigned)kCellK) R.slot[c * kCellK + slot_k] = (uint16_t)i;
        else ok = false;
    }
    __syncwarp();
    ok = __all_sync(0xffffffffu, ok);
    if (!ok) {
        for (int c = lane; c < ncell; c += 32)
            if (R.cnt[c] > kCellK) R.cnt[c] = (uint8_t)kCellK;
        __syncwarp();
    }
    return ok;
}

// Visit the squares of the 3x3 cell block around (cx, cy): returns through
// `fn(j)` for every candidate t = lane, lane + kStride, ... (kStride lanes
// share the block: the whole warp, or one half of it).
template <int kStride = 32, typename Fn>
__device__ __forceinline__ void for_block(const Rep& R, const Grid& g, int cx, int cy, int lane, Fn&& fn) {
    // Every lane reads the nine cell counts (broadcast shared loads) and
    // forms their running sum; slot t of the block belongs to the first cell
    // whose running count exceeds t.  Lanes take slots 32 apart.  The cell
    // of slot t is rebuilt from (cx, cy) and its index in the block, so no
    // per-lane array is indexed at run time.
    int ends[9];
    int run = 0;
#pragma unroll
    for (int c = 0; c < 9; ++c) {
        const int x = cx + c % 3 - 1, y = cy + c / 3 - 1;
        const bool in = (unsigned)x < (unsigned)g.G && (unsigned)y < (unsigned)g.G;
        run += in ? (int)R.cnt[y * g.G + x] : 0;
        ends[c] = run;
    }
    for (int t = lane; t < run; t += kStride) {
        int c = 0, start = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const bool past = t >= ends[k];
            c = past ? k + 1 : c;
            start = past ? ends[k] : start;
        }
        const int cr = (c * 43) >> 7;  // c / 3 for c < 9
        const int cell = (cy + cr - 1) * g.G + cx + (c - 3 * cr) - 1;
        fn((int)R.slot[cell * kCellK + (t - start)]);
    }
}

// Warp sum of the fixed-point energy change of one proposal: each lane's
// term is split as hi * 2^20 + lo (0 <= lo < 2^20) and both parts are summed
// with 32-bit warp reductions.  Exact while every lane's term is below 2^46
// in magnitude: a proposal's lane holds a few pair terms of at most
// 1.5 * 2^40 each (and lane 0 the wall change), far inside that.
__device__ __forceinline__ long long warp_sum_dq(long long v) {
    const unsigned lo = (unsigned)(v & 0xFFFFF);
    const int hi = (int)(v >> 20);
    const unsigned slo = __reduce_add_sync(0xffffffffu, lo);
    const int shi = __reduce_add_sync(0xffffffffu, hi);
    return (long long)shi * 1048576ll + (long long)slo;
}

__device__ __forceinline__ long long qe(float e) { return __float2ll_rn(e * kEScale); }

// Change of square Q's pair term when a square moves from P to (nx, ny) with
// (cos, sin) = (nc, ns), in kEScale units.  Both terms are evaluated and each
// is kept only inside the cut-off: the same values as testing first, without
// a branch around them (a warp's lanes almost always disagree on the test).
__device__ __forceinline__ long long pair_delta(float4 Q, float nx, float ny, float nc, float ns, float4 P) {
    const float ex = Q.x - nx, ey = Q.y - ny, fx = Q.x - P.x, fy = Q.y - P.y;
    const long long en = qe(sat_pair_energy(ex, ey, nc, ns, Q.z, Q.w));
    const long long eo = qe(sat_pair_energy(fx, fy, P.z, P.w, Q.z, Q.w));
    return (ex * ex + ey * ey < kPairCut2 ? en : 0) - (fx * fx + fy * fy < kPairCut2 ? eo : 0);
}

__device__ __forceinline__ long long warp_sum_ll(long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_max_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ double warp_min_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Full energy of one replica (walls + each neighbour pair once), fixed point.
__device__ long long full_energy(const Rep& R, int n, const Grid& g, float L, int lane) {
    long long e = 0;
    for (int i = 0; i < n; ++i) {
        const float4 P = R.sq[i];
        if (lane == 0) e += qe(wall_e(P.x, P.y, P.z, P.w, L));
        for_block(R, g, g.cx(P.x), g.cx(P.y), lane, [&](int j) {
            if (j > i) {
                const float4 Q = R.sq[j];
                const float dx = Q.x - P.x, dy = Q.y - P.y;
                if (dx * dx + dy * dy < kPairCut2) e += qe(sat_pair_energy(dx, dy, P.z, P.w, Q.z, Q.w));
            }
        });
    }
    return warp_sum_ll(e);
}

// FP64 dilation-certified side of a replica (device_certified_side,
// seeded.cu:175-226): the smallest centre dilation lambda that opens a
// tau = 2.6e-8 gap along the best axis of every close pair, rejection above
// 1.008, side of the bounding box of the dilated squares.  Products are kept
// unfused so the result rounds like the host oracle's.
__device__ double cert_side(const Rep& R, int n, const Grid& g, int lane, double& lam_out, double& x0_out,
                            double& y0_out) {
    const double tau = 2.6e-8;
    double lam = 1.0;
    for (int i = lane; i < n; i += 32) {
        const float4 P = R.sq[i];
        const double xi = P.x, yi = P.y;
        double si, ci;
        sincos((double)R.ang[i], &si, &ci);
        const int cx = g.cx(P.x), cy = g.cx(P.y);
        for (int dy = -1; dy <= 1; ++dy) {
            for (int dxc = -1; dxc <= 1; ++dxc) {
                const int x = cx + dxc, y = cy + dy;
                if (x < 0 || x >= g.G || y < 0 || y >= g.G) continue;
                const int cell = y * g.G + x;
                const int m = R.cnt[cell];
                for (int k = 0; k < m; ++k) {
                    const int j = R.slot[cell * kCellK + k];
                    if (j <= i) continue;
                    const double dx = __dsub_rn(xi, (double)R.sq[j].x), dyv = __dsub_rn(yi, (double)R.sq[j].y);
                    if (__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dyv, dyv)) >= 2.05) continue;
                    double sj, cj;
                    sincos((double)R.ang[j], &sj, &cj);
                    const double c12 = fabs(__dadd_rn(__dmul_rn(ci, cj), __dmul_rn(si, sj)));
                    const double s12 = fabs(__dadd_rn(__dmul_rn(-si, cj), __dmul_rn(ci, sj)));
                    const double r = __dadd_rn(0.5, __dmul_rn(0.5, __dadd_rn(c12, s12)));
                    const double v1 = fabs(__dadd_rn(__dmul_rn(dx, ci), __dmul_rn(dyv, si)));
                    const double v2 = fabs(__dadd_rn(__dmul_rn(-dx, si), __dmul_rn(dyv, ci)));
                    const double v3 = fabs(__dadd_rn(__dmul_rn(dx, cj), __dmul_rn(dyv, sj)));
                    const double v4 = fabs(__dadd_rn(__dmul_rn(-dx, sj), __dmul_rn(dyv, cj)));
                    const double vmax = fmax(fmax(v1, v2), fmax(v3, v4));
                    const double req = vmax > 1e-12 ? __ddiv_rn(__dadd_rn(r, tau), vmax) : 1e9;
                    lam = fmax(lam, req);
                }
            }
        }
    }
    lam = warp_max_d(lam);
    lam_out = lam;
    if (lam > 1.008) return 1e9;
    double bx0 = 1e9, bx1 = -1e9, by0 = 1e9, by1 = -1e9;
    for (int i = lane; i < n; i += 32) {
        const float4 P = R.sq[i];
        const double x = __dmul_rn((double)P.x, lam), y = __dmul_rn((double)P.y, lam);
        double s, c;
        sincos((double)R.ang[i], &s, &c);
        const double r = __dmul_rn(0.5, __dadd_rn(fabs(c), fabs(s)));
        bx0 = fmin(bx0, __dsub_rn(x, r));
        bx1 = fmax(bx1, __dadd_rn(x, r));
        by0 = fmin(by0, __dsub_rn(y, r));
        by1 = fmax(by1, __dadd_rn(y, r));
    }
    bx0 = warp_min_d(bx0);
    bx1 = warp_max_d(bx1);
    by0 = warp_min_d(by0);
    by1 = warp_max_d(by1);
    x0_out = bx0;
    y0_out = by0;
    return fmax(__dsub_rn(bx1, bx0), __dsub_rn(by1, by0));
}

__device__ long long block_sum_ll(long long v, long long* red);

// Three sums at once over the warps w < nw of a group whose warp partials
// go to red[3 w .. 3 w + 2]; `sync` orders the slots' writes and reads.
template <class Sync>
__device__ __forceinline__ void group_sum3(long long& a, long long& b, long long& c, long long* red, int wg, int nw,
                                           Sync&& sync) {
    a = warp_sum_ll(a);
    b = warp_sum_ll(b);
    c = warp_sum_ll(c);
    sync();
    if ((threadIdx.x & 31) == 0) {
        red[3 * wg] = a;
        red[3 * wg + 1] = b;
        red[3 * wg + 2] = c;
    }
    sync();
    a = b = c = 0;
    for (int k = 0; k < nw; ++k) {
        a += red[3 * k];
        b += red[3 * k + 1];
        c += red[3 * k + 2];
    }
}

// ---- Cooperative forms: a group of threads works on one replica, either
// the whole CTA (CtaGrp) or one warp (WarpGrp).  Results do not depend on the
// group: every sum below is an integer sum and slot order within a cell list
// changes no energy, gradient or decision.
struct CtaGrp {
    long long* red;  // one slot per warp of the CTA
    __device__ __forceinline__ int t() const { return threadIdx.x; }
    __device__ __forceinline__ int nt() const { return blockDim.x; }
    __device__ __forceinline__ void sync() const { __syncthreads(); }
    __device__ __forceinline__ bool sync_or(bool p) const { return __syncthreads_or(p); }
    __device__ __forceinline__ long long sum(long long v) const { return block_sum_ll(v, red); }
    __device__ __forceinline__ void sum3(long long& a, long long& b, long long& c) const {
        group_sum3(a, b, c, red, (int)threadIdx.x >> 5, (int)(blockDim.x + 31) >> 5, [] { __syncthreads(); });
    }
};
struct WarpGrp {
    int lane;
    __device__ __forceinline__ int t() const { return lane; }
    __device__ __forceinline__ int nt() const { return 32; }
    __device__ __forceinline__ void sync() const { __syncwarp(); }
    __device__ __forceinline__ bool sync_or(bool p) const {
        __syncwarp();
        return __any_sync(0xffffffffu, p);
    }
    __device__ __forceinline__ long long sum(long long v) const { return warp_sum_ll(v); }
    __device__ __forceinline__ void sum3(long long& a, long long& b, long long& c) const {
        a = warp_sum_ll(a);
        b = warp_sum_ll(b);
        c = warp_sum_ll(c);
    }
};
// `nw` consecutive warps of the CTA (nw >= 2) on named barrier `id` (1..15).
struct BarGrp {
    int id, nw, t0;  // barrier, warps, first thread of the group
    long long* red;  // three slots per warp of the group
    __device__ __forceinline__ int t() const { return (int)threadIdx.x - t0; }
    __device__ __forceinline__ int nt() const { return 32 * nw; }
    __device__ __forceinline__ void sync() const {
        asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(32 * nw) : "memory");
    }
    __device__ __forceinline__ bool sync_or(bool p) const {
        unsigned r;
        asm volatile(
            "{\n\t.reg .pred ip, op;\n\tsetp.ne.u32 ip, %1, 0;\n\tbar.red.or.pred op, %2, %3, ip;\n\t"
            "selp.u32 %0, 1, 0, op;\n\t}"
            : "=r"(r)
            : "r"((unsigned)p), "r"(id), "r"(32 * nw)
            : "memory");
        return r != 0;
    }
    __device__ __forceinline__ long long sum(long long v) const {
        v = warp_sum_ll(v);
        sync();  // every read of the slots by the previous sum is done
        if ((threadIdx.x & 31) == 0) red[t() >> 5] = v;
        sync();
        long long s = 0;
        for (int k = 0; k < nw; ++k) s += red[k];
        return s;
    }
    __device__ __forceinline__ void sum3(long long& a, long long& b, long long& c) const {
        group_sum3(a, b, c, red, t() >> 5, nw, [this] { sync(); });
    }
};

template <class Grp>
__device__ bool build_cells_grp(const Grp& gp, const Rep& R, int n, const Grid& g) {
    const int ncell = g.G * g.G, tid = gp.t(), nt = gp.nt();
    for (int c = tid; c < ncell; c += nt) R.cnt[c] = 0;
    for (int k = tid; k < ncell * kCellK; k += nt) R.slot[k] = 0;
    gp.sync();
    bool ok = true;
    for (int i = tid; i < n; i += nt) {
        const float4 p = R.sq[i];
        const int c = g.cx(p.y) * g.G + g.cx(p.x);
        const unsigned k = atomicAdd(reinterpret_cast<unsigned*>(R.cnt + (c & ~3)), 1u << (8 * (c & 3)));
        const unsigned slot_k = (k >> (8 * (c & 3))) & 0xffu;
        if (slot_k < (unsigned)kCellK) R.slot[c * kCellK + slot_k] = (uint16_t)i;
        else ok = false;
    }
    const bool bad = gp.sync_or(!ok);
    if (bad) {
        for (int c = tid; c < ncell; c += nt)
            if (R.cnt[c] > kCellK) R.cnt[c] = (uint8_t)kCellK;
        gp.sync();
    }
    return !bad;
}

__device__ long long block_sum_ll(long long v, long long* red) {
    v = warp_sum_ll(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    long long t = 0;
    for (int k = 0; k < nw; ++k) t += red[k];
    return t;
}

// Full fixed-point energy by the whole CTA.  Work item w is square w / 9
// against the squares listed in cell w % 9 of its 3 x 3 block (each pair
// counted from its lower index), so a small replica still spreads over
// many threads.
template <class Grp>
__device__ long long full_energy_grp(const Grp& gp, const Rep& R, int n, const Grid& g, float L) {
    long long e = 0;
    for (int w = gp.t(); w < 9 * n; w += gp.nt()) {
        const int i = w / 9, c = w - 9 * i;
        const float4 P = R.sq[i];
        if (c == 0) e += qe(wall_e(P.x, P.y, P.z, P.w, L));
        const int x = g.cx(P.x) + c % 3 - 1, y = g.cx(P.y) + c / 3 - 1;
        if (x < 0 || x >= g.G || y < 0 || y >= g.G) continue;
        const int cell = y * g.G + x, m = R.cnt[cell];
        for (int k = 0; k < m; ++k) {
            const int j = R.slot[cell * kCellK + k];
            if (j <= i) continue;
            const float4 Q = R.sq[j];
            const float dx = Q.x - P.x, dy2 = Q.y - P.y;
            if (dx * dx + dy2 * dy2 < kPairCut2) e += qe(sat_pair_energy(dx, dy2, P.z, P.w, Q.z, Q.w));
        }
    }
    return gp.sum(e);
}

// Quench gradient sums: 32-bit integers in units of 2^-20.  A square's 3 x 3
// block lists at most 9 x 12 partners, each term below 5.2 (and the wall
// term below 1), so a sum stays below 6e8 < 2^31; integer atomics make the
// sums independent of the order of the terms.
constexpr float kQScale = 1048576.0f;
__device__ __forceinline__ int qg(float v) { return __float2int_rn(v * kQScale); }

// Line-search pair list.  A trial moves every centre coordinate by at most
// kListStep from the saved state; then a pair within the cut-off at the trial
// was at most 1.4142 + 2 kListStep < 1.59 (the smallest cell side) apart per
// axis at the saved state, so it sits in the saved 3 x 3 cell blocks, and at
// most sqrt(kPairCut2) + 2 sqrt(2) kListStep = 1.6546 apart: the pairs of
// those blocks closer than sqrt(kListCut2) = 1.6583 hold every pair with a
// non-zero trial energy, and the list's energy equals the full one exactly.
constexpr float kListStep = 0.085f, kListCut2 = 2.75f;

template <class Grp>
__device__ long long list_energy(const Grp& gp, const Rep& R, int n, float L, const uint32_t* pl, int cnt) {
    long long e = 0;
    for (int i = gp.t(); i < n; i += gp.nt()) {
        const float4 P = R.sq[i];
        e += qe(wall_e(P.x, P.y, P.z, P.w, L));
    }
    for (int k = gp.t(); k < cnt; k += gp.nt()) {
        const uint32_t pr = pl[k];
        const float4 P = R.sq[pr & 0xffffu], Q = R.sq[pr >> 16];
        const float dx = Q.x - P.x, dy = Q.y - P.y;
        if (dx * dx + dy * dy < kPairCut2) e += qe(sat_pair_energy(dx, dy, P.z, P.w, Q.z, Q.w));
    }
    return gp.sum(e);
}

__device__ __forceinline__ long long clamp_q24(int v) { return max(-(1 << 24), min(1 << 24, v)); }

// The checkpoint quench of one replica (the coldest, or each one under
// SQS_JOB_QUENCH_ALL) by a group of threads: the reference's conjugate-gradient
// polish (seeded.cu:621-715) on the overlap energy.  Each iteration takes the
// gradient (one thread per (square, neighbouring cell) work item), a
// Polak-Ribiere direction d = -g + beta d (beta = max(0, (g - g_old).g /
// g_old.g), 0 on the first iteration and every 25th), and a backtracking
// line search of up to 5 trials from the carried step (x 0.45 per trial).
// An accepted trial sets the step to min(0.15, 1.25 alpha); when no trial
// improves, the state goes back, the direction is dropped and the step
// halves (at least 1e-7) -- the polish goes on, it does not stop there.  It
// ends at zero energy, at a zero gradient, after `iters` iterations, or, with
// a stall limit (not kQuenchNoStall), after `stall_limit` accepted steps in a
// row that each gained less than 0.1% or at a line search without a gain.
// Gradients and their dot products are integer sums, so the result does not
// depend on the group's width.  Scratch: kQuenchScr n float4 (gradient sums,
// previous gradient, direction, saved state, pair list: a counter, the
// largest direction component and up to 8 n - 2 pairs).
template <class Grp>
__device__ long long quench_grp(const Grp& gp, const Rep& R, int n, const Grid& g, float L, int iters, int stall_limit,
                                float4* scr, long long E) {
    int4* acc = reinterpret_cast<int4*>(scr);       // gradient sums of this iteration
    int4* gold = reinterpret_cast<int4*>(scr + n);  // the previous iteration's
    float4* dir = scr + 2 * n;                      // search direction
    float4* saved = scr + 3 * n;                    // state before the line search
    uint32_t* plist = reinterpret_cast<uint32_t*>(scr + 4 * n);  // [0] count, [1] max |d|, pairs
    const int pcap = 8 * n - 2;
    float step = 0.04f;
    int stall = 0;  // consecutive accepted steps that gained less than 0.1%
    float drift = 1e30f;  // bound on any centre's per-axis move since the pair list was built (none yet)
    for (int i = gp.t(); i < n; i += gp.nt()) {
        gold[i] = make_int4(0, 0, 0, 0);
        dir[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    for (int it = 0; it < iters && E > 0; ++it) {
        for (int i = gp.t(); i < n; i += gp.nt()) {
            acc[i] = make_int4(0, 0, 0, 0);
            saved[i] = make_float4(R.sq[i].x, R.sq[i].y, R.ang[i], 0.f);
        }
        // the pair list stays exact while no centre has moved more than
        // kListStep per axis since it was built; past that it is rebuilt
        const bool rebuild = !(drift <= kListStep);
        if (gp.t() == 0) {
            if (rebuild) plist[0] = 0u;
            plist[1] = 0u;
        }
        gp.sync();
        if (!rebuild) {
            // gradient over the list: walls, then both sides of every pair
            // within the cut-off (the cell scan's operations and sums)
            for (int i = gp.t(); i < n; i += gp.nt()) {
                const float4 P = R.sq[i];
                float wx = 0.f, wy = 0.f, wa = 0.f;
                wall_energy_grad(P.x, P.y, P.z, P.w, L, wx, wy, wa);
                const int ax = qg(wx), ay = qg(wy), aa = qg(wa);
                if (ax | ay | aa) {
                    atomicAdd(&acc[i].x, ax);
                    atomicAdd(&acc[i].y, ay);
                    atomicAdd(&acc[i].z, aa);
                }
            }
            const int np = (int)plist[0];
            for (int k = gp.t(); k < np; k += gp.nt()) {
                const uint32_t pr = plist[2 + k];
                const int i = (int)(pr & 0xffffu), j = (int)(pr >> 16);
                const float4 P = R.sq[i], Q = R.sq[j];
                const float ex = Q.x - P.x, ey = Q.y - P.y;
                if (ex * ex + ey * ey >= kPairCut2) continue;
                PairGrad pg;
                if (sat_pair_grad(ex, ey, P.z, P.w, Q.z, Q.w, pg)) {
                    atomicAdd(&acc[i].x, qg(pg.px));
                    atomicAdd(&acc[i].y, qg(pg.py));
                    atomicAdd(&acc[i].z, qg(pg.pa));
                }
                if (sat_pair_grad(P.x - Q.x, P.y - Q.y, Q.z, Q.w, P.z, P.w, pg)) {
                    atomicAdd(&acc[j].x, qg(pg.px));
                    atomicAdd(&acc[j].y, qg(pg.py));
                    atomicAdd(&acc[j].z, qg(pg.pa));
                }
            }
        }
        // work item w: square w / 9 against cell w % 9 of its block; it also
        // lists the block's pairs (i < j) closer than sqrt(kListCut2)
        for (int w = gp.t(); rebuild && w < 9 * n; w += gp.nt()) {
            const int i = w / 9, c = w - 9 * i;
            const float4 P = R.sq[i];
            int ax = 0, ay = 0, aa = 0;
            if (c == 0) {
                float wx = 0.f, wy = 0.f, wa = 0.f;
                wall_energy_grad(P.x, P.y, P.z, P.w, L, wx, wy, wa);
                ax = qg(wx);
                ay = qg(wy);
                aa = qg(wa);
            }
            const int x = g.cx(P.x) + c % 3 - 1, y = g.cx(P.y) + c / 3 - 1;
            if (x >= 0 && x < g.G && y >= 0 && y < g.G) {
                const int cell = y * g.G + x, m = R.cnt[cell];
                for (int k = 0; k < m; ++k) {
                    const int j = R.slot[cell * kCellK + k];
                    if (j == i) continue;
                    const float4 Q = R.sq[j];
                    const float ex = Q.x - P.x, ey = Q.y - P.y;
                    const float d2 = ex * ex + ey * ey;
                    if (j > i && d2 < kListCut2) {
                        const uint32_t slot = atomicAdd(&plist[0], 1u);
                        if (slot < (uint32_t)pcap) plist[2 + slot] = (uint32_t)i | ((uint32_t)j << 16);
                    }
                    if (d2 >= kPairCut2) continue;
                    PairGrad pg;
                    if (sat_pair_grad(ex, ey, P.z, P.w, Q.z, Q.w, pg)) {
                        ax += qg(pg.px);
                        ay += qg(pg.py);
                        aa += qg(pg.pa);
                    }
                }
            }
            if (ax | ay | aa) {
                atomicAdd(&acc[i].x, ax);
                atomicAdd(&acc[i].y, ay);
                atomicAdd(&acc[i].z, aa);
            }
        }
        gp.sync();
        if (rebuild) drift = plist[0] <= (uint32_t)pcap ? 0.f : 1e30f;  // an overflowed list is not used
        // Polak-Ribiere: g_old.g_old, (g - g_old).g and g.g as exact integer
        // sums of components clamped to 2^24 (a gradient of 16; only beta
        // sees the clamp): 3 n <= 3000 terms below 2^49 each fit 64 bits
        long long s_oo = 0, s_dg = 0, s_gg = 0;
        for (int i = gp.t(); i < n; i += gp.nt()) {
            const int4 a = acc[i], o = gold[i];
            const long long gx = clamp_q24(a.x), gy = clamp_q24(a.y), ga = clamp_q24(a.z);
            const long long ox = clamp_q24(o.x), oy = clamp_q24(o.y), oa = clamp_q24(o.z);
            s_oo += ox * ox + oy * oy + oa * oa;
            s_dg += (gx - ox) * gx + (gy - oy) * gy + (ga - oa) * ga;
            s_gg += gx * gx + gy * gy + ga * ga;
        }
        gp.sum3(s_oo, s_dg, s_gg);
        const float beta =
            (it == 0 || s_oo == 0 || it % 25 == 0) ? 0.f : fmaxf(0.f, (float)((double)s_dg / (double)s_oo));
        if (s_gg == 0 && beta == 0.f) break;  // no direction left at the sums' resolution
        uint32_t dmax_bits = 0u;  // largest |d.x|, |d.y| (bits of non-negative floats order as integers)
        for (int i = gp.t(); i < n; i += gp.nt()) {
            const int4 a = acc[i];
            const float4 d0 = dir[i];
            const float4 d1 = make_float4(__fmaf_rn(beta, d0.x, -(float)a.x * (1.0f / kQScale)),
                                          __fmaf_rn(beta, d0.y, -(float)a.y * (1.0f / kQScale)),
                                          __fmaf_rn(beta, d0.z, -(float)a.z * (1.0f / kQScale)), 0.f);
            dir[i] = d1;
            gold[i] = a;
            dmax_bits = max(dmax_bits, __float_as_uint(fmaxf(fabsf(d1.x), fabsf(d1.y))));
        }
        dmax_bits = __reduce_max_sync(0xffffffffu, dmax_bits);
        if ((threadIdx.x & 31) == 0) atomicMax(&plist[1], dmax_bits);
        gp.sync();
        const int npairs = (int)plist[0];
        const float dmax = __uint_as_float(plist[1]);
        // Trial steps move every coordinate by at most 0.1, so each partner
        // within the pair cut-off of a moved square still sits in one of the
        // 3 x 3 cells around it on the lists built for the saved state
        // (1.4142 + 0.1 < 1.59 <= cell side): trial energies use those lists,
        // and the lists are rebuilt only for an accepted step.  A trial that
        // keeps every centre within kListStep per axis of where the pair list
        // was built sums the list instead (the same energy, without the cell
        // scan).
        float alpha = step;
        bool moved = false;
        for (int tries = 0; tries < 5 && !moved; ++tries) {
            for (int i = gp.t(); i < n; i += gp.nt()) {
                const float4 d = dir[i], o = saved[i];
                const float sx = fminf(0.1f, fmaxf(-0.1f, alpha * d.x));
                const float sy = fminf(0.1f, fmaxf(-0.1f, alpha * d.y));
                float a = o.z + fminf(0.1f, fmaxf(-0.1f, alpha * d.z));
                a = a - kHalfPiF * floorf(a * (1.0f / kHalfPiF));
                if (!(a >= 0.f && a < kHalfPiF)) a = 0.f;
                float sn, cs;
                state_trig(a, &sn, &cs);
                R.sq[i] = make_float4(o.x + sx, o.y + sy, cs, sn);
                R.ang[i] = a;
            }
            gp.sync();
            const bool by_list = npairs <= pcap && drift + alpha * dmax <= kListStep;
            const long long En = by_list ? list_energy(gp, R, n, L, plist + 2, npairs) : full_energy_grp(gp, R, n, g, L);
            if (En < E && build_cells_grp(gp, R, n, g)) {
                stall = En > E - E / 1000 ? stall + 1 : 0;  // less than 0.1% gained
                E = En;
                step = fminf(0.15f, alpha * 1.25f);
                drift += fminf(0.1f, alpha * dmax);  // every centre moved at most this far per axis
                moved = true;
            } else {
                if (En < E) {  // the better state overflows a cell: lists back to the saved state
                    for (int i = gp.t(); i < n; i += gp.nt()) {
                        const float4 o = saved[i];
                        float sn, cs;
                        state_trig(o.z, &sn, &cs);
                        R.sq[i] = make_float4(o.x, o.y, cs, sn);
                        R.ang[i] = o.z;
                    }
                    gp.sync();
                    build_cells_grp(gp, R, n, g);  // the saved state fitted
                }
                alpha *= 0.45f;
            }
        }
        if (!moved) {  // back to the saved state (its lists are current), direction dropped
            for (int i = gp.t(); i < n; i += gp.nt()) {
                const float4 o = saved[i];
                float sn, cs;
                state_trig(o.z, &sn, &cs);
                R.sq[i] = make_float4(o.x, o.y, cs, sn);
                R.ang[i] = o.z;
                dir[i] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
            step = fmaxf(1e-7f, step * 0.5f);
            gp.sync();
            if (stall_limit < kQuenchNoStall) break;  // the library's default quench ends here
        }
        if (stall >= stall_limit) break;
    }
    return E;
}

__device__ __forceinline__ float wrap_quarter_f(float a) {
    a = a - kHalfPiF * floorf(a * (1.0f / kHalfPiF));
    return (a >= 0.f && a < kHalfPiF) ? a : 0.f;
}

// Collective proposal (one warp, one replica): the set of squares the mode
// selects around square `c` -- 1 its row (|dy| < 0.55), 2 its column
// (|dx| < 0.55), 3 the disc dx^2 + dy^2 < 2.5, 4 its orientation class
// (angles within 0.06 modulo pi/2), 5 its diagonal strips (|dx +- dy| < 0.85),
// 6 every tilted square (0.04 < a < 1.53) -- is translated by (tx, ty)
// (mode 6: by +-(tx, ty) alternating with the square index), rotated about
// the drawn square by `th` for modes 3 and 4, and every moved square turned by
// `th` (seeded.cu:547-613).  Centres stay in [0.5, L - 0.5].  The move is
// judged on the full fixed-point energy; a rejected move (or one that
// overflows a cell) is undone from `save`, the replica's own HBM slot, which
// holds nothing else while a slice runs.  Returns whether it was accepted;
// *ovf counts overflows.
__device__ __forceinline__ bool collective_move(const Rep& rep, const Grid& g, int n, float L, int lane, int mode, int c,
                                             float tx, float ty, float th, float u, float invT, long long& E,
                                             float4* __restrict__ save, int* ovf) {
    const float cx = rep.sq[c].x, cy = rep.sq[c].y, ca = rep.ang[c];
    float st, ct;
    state_trig(th, &st, &ct);
    __syncwarp();
    for (int s = lane; s < n; s += 32) {
        const float4 P = rep.sq[s];
        const float a = rep.ang[s];
        const float ex = P.x - cx, ey = P.y - cy, da = a - ca;
        const bool take = mode == 1   ? fabsf(ey) < 0.55f
                          : mode == 2 ? fabsf(ex) < 0.55f
                          : mode == 3 ? ex * ex + ey * ey < 2.5f
                          : mode == 4 ? (fabsf(da) < 0.06f || fabsf(da) > kHalfPiF - 0.06f)
                          : mode == 5 ? (fabsf(ex + ey) < 0.85f || fabsf(ex - ey) < 0.85f)
                                      : (a > 0.04f && a < 1.53f);
        save[s] = make_float4(P.x, P.y, a, take ? 1.f : 0.f);
        if (take) {
            float nx, ny;
            if (mode == 3 || mode == 4) {
                nx = cx + ct * ex - st * ey + tx;
                ny = cy + st * ex + ct * ey + ty;
            } else if (mode == 6) {
                const float sg = (s & 1) ? 1.f : -1.f;
                nx = P.x + sg * tx;
                ny = P.y + sg * ty;
            } else {
                nx = P.x + tx;
                ny = P.y + ty;
            }
            nx = fminf(L - 0.5f, fmaxf(0.5f, nx));
            ny = fminf(L - 0.5f, fmaxf(0.5f, ny));
            const float na = wrap_quarter_f(a + th);
            float sn, cs;
            state_trig(na, &sn, &cs);
            rep.sq[s] = make_float4(nx, ny, cs, sn);
            rep.ang[s] = na;
        }
    }
    __syncwarp();
    const bool fits = build_cells(rep, n, g, lane);
    bool acc = false;
    if (fits) {
        const long long En = full_energy(rep, n, g, L, lane);
        const long long dq = En - E;
        acc = dq <= 0 || u < __expf(-((float)dq * (1.0f / kEScale)) * invT);
        if (acc) E = En;
    } else {
        ++*ovf;
    }
    if (!acc) {
        for (int s = lane; s < n; s += 32) {
            const float4 o = save[s];
            if (o.w != 0.f) {
                float sn, cs;
                state_trig(o.z, &sn, &cs);
                rep.sq[s] = make_float4(o.x, o.y, cs, sn);
                rep.ang[s] = o.z;
            }
        }
        __syncwarp();
        build_cells(rep, n, g, lane);  // the saved state fitted
    }
    return acc;
}

// Kick of an overlapped replica at an exchange round (seeded.cu:721-778):
// every square's energy (its wall term and its pairs); on odd rounds, when
// the worst square's energy exceeds 1e-5, that square moves to the probe of
// an 8 x 8 grid over [0.55, L - 0.55]^2 farthest from every other centre
// (jittered by up to 0.05, a fresh angle); then every square is jittered,
// by up to 0.08 / 0.18 rad where its energy exceeds 1e-6 and 0.008 / 0.015
// elsewhere.  Draws are Philox blocks keyed by (round, square, replica).
// Returns the new energy (the old one if a cell would overflow, the state
// then restored from `save`).
__device__ __forceinline__ long long kick_replica(const Rep& rep, const Grid& g, int n, float L, int lane, int r,
                                               int round, uint32_t k0, uint32_t k1, long long E,
                                               float4* __restrict__ save) {
    float wmax = -1.f;
    int worst = 0x7fffffff;
    for (int s = lane; s < n; s += 32) {
        const float4 P = rep.sq[s];
        float e = wall_e(P.x, P.y, P.z, P.w, L);
        const int cxs = g.cx(P.x), cys = g.cx(P.y);
        for (int dyc = -1; dyc <= 1; ++dyc) {
            for (int dxc = -1; dxc <= 1; ++dxc) {
                const int x = cxs + dxc, y = cys + dyc;
                if (x < 0 || x >= g.G || y < 0 || y >= g.G) continue;
                const int cell = y * g.G + x, m = rep.cnt[cell];
                for (int k = 0; k < m; ++k) {
                    const int j = rep.slot[cell * kCellK + k];
                    if (j == s) continue;
                    const float4 Q = rep.sq[j];
                    const float dx = Q.x - P.x, dy = Q.y - P.y;
                    if (dx * dx + dy * dy < kPairCut2) e += sat_pair_energy(dx, dy, P.z, P.w, Q.z, Q.w);
                }
            }
        }
        save[s] = make_float4(P.x, P.y, rep.ang[s], e);
        if (e > wmax) {
            wmax = e;
            worst = s;
        }
    }
    // warp arg-max (ties: the smaller index)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float om = __shfl_xor_sync(0xffffffffu, wmax, o);
        const int oi = __shfl_xor_sync(0xffffffffu, worst, o);
        if (om > wmax || (om == wmax && oi < worst)) {
            wmax = om;
            worst = oi;
        }
    }
    if ((round & 1) && wmax > 1e-5f && worst < n) {
        float bd = -1.f;
        int bp = 64;
        for (int p = lane; p < 64; p += 32) {
            const float vx = 0.55f + (L - 1.1f) * ((float)(p % 8) + 0.5f) / 8.f;
            const float vy = 0.55f + (L - 1.1f) * ((float)(p / 8) + 0.5f) / 8.f;
            float d2 = 1e9f;
            for (int j = 0; j < n; ++j) {
                if (j == worst) continue;
                const float dx = vx - rep.sq[j].x, dy = vy - rep.sq[j].y;
                d2 = fminf(d2, dx * dx + dy * dy);
            }
            if (d2 > bd) {
                bd = d2;
                bp = p;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float od = __shfl_xor_sync(0xffffffffu, bd, o);
            const int op = __shfl_xor_sync(0xffffffffu, bp, o);
            if (od > bd || (od == bd && op < bp)) {
                bd = od;
                bp = op;
            }
        }
        if (lane == 0) {
            const U4 q = philox4x32_10(U4{(uint32_t)round, 0xffffu, (uint32_t)r, 3u}, k0, k1);
            const float vx = 0.55f + (L - 1.1f) * ((float)(bp % 8) + 0.5f) / 8.f;
            const float vy = 0.55f + (L - 1.1f) * ((float)(bp / 8) + 0.5f) / 8.f;
            const float na = wrap_quarter_f(u01(q.z) * kHalfPiF);
            float sn, cs;
            state_trig(na, &sn, &cs);
            rep.sq[worst] = make_float4(fminf(L - 0.5f, fmaxf(0.5f, vx + 0.05f * (2.f * u01(q.x) - 1.f))),
                                        fminf(L - 0.5f, fmaxf(0.5f, vy + 0.05f * (2.f * u01(q.y) - 1.f))), cs, sn);
            rep.ang[worst] = na;
        }
        __syncwarp();
    }
    for (int s = lane; s < n; s += 32) {
        const float hot = save[s].w > 1e-6f;
        const float axy = hot ? 0.08f : 0.008f, aa = hot ? 0.18f : 0.015f;
        const U4 q = philox4x32_10(U4{(uint32_t)round, (uint32_t)s, (uint32_t)r, 2u}, k0, k1);
        const float4 P = rep.sq[s];
        const float na = wrap_quarter_f(rep.ang[s] + aa * (2.f * u01(q.z) - 1.f));
        float sn, cs;
        state_trig(na, &sn, &cs);
        rep.sq[s] = make_float4(fminf(L - 0.48f, fmaxf(0.48f, P.x + axy * (2.f * u01(q.x) - 1.f))),
                                fminf(L - 0.48f, fmaxf(0.48f, P.y + axy * (2.f * u01(q.y) - 1.f))), cs, sn);
        rep.ang[s] = na;
    }
    __syncwarp();
    if (build_cells(rep, n, g, lane)) return full_energy(rep, n, g, L, lane);
    for (int s = lane; s < n; s += 32) {
        const float4 o = save[s];
        float sn, cs;
        state_trig(o.z, &sn, &cs);
        rep.sq[s] = make_float4(o.x, o.y, cs, sn);
        rep.ang[s] = o.z;
    }
    __syncwarp();
    build_cells(rep, n, g, lane);
    return E;
}

// Rungs per ladder (a job's R rungs form `ladders` ladders of RL rungs; rung
// k is position k % RL of ladder k / RL, as the reference groups its chains
// into ladders of 8, seeded.cu:493, 791-817).
__device__ __forceinline__ int rungs_per_ladder(const JobDev& jd) { return jd.R / max(1, jd.ladders); }

// Ladder temperature of rung k: geometric from tmin (position 0) to tmax
// (position RL - 1), the reference's ladder T_b = tmin (tmax / tmin)^(b / 7)
// for RL = 8 (seeded.cu:493-494).
__device__ __forceinline__ float rung_temp(const JobDev& jd, int k) {
    const int RL = rungs_per_ladder(jd), pos = k % RL;
    const float lt = logf(jd.tmin), lh = logf(jd.tmax);
    return RL > 1 ? expf(lt + (lh - lt) * (float)pos / (float)(RL - 1)) : jd.tmin;
}

// Cooling factor of exchange round x under SQS_JOB_ADAPT: 0.002^((x mod 200)
// / 199), the reference's cool (seeded.cu:493); 1 otherwise.
__device__ __forceinline__ float cool_of(bool adaptive, int xround) {
    return adaptive ? powf(0.002f, (float)(xround % 200) / 199.f) : 1.f;
}

// Step scale of a replica on rung k under SQS_JOB_ADAPT: adaptation factor x
// (0.15 + 1.85 pos / (RL - 1)) x sqrt(cool), the reference's scale = adapt *
// baseMove * (.15 + 1.85 (b % 8) / 7) * sqrt(cool) (seeded.cu:506), in units
// of the job's sigma.
__device__ __forceinline__ float step_scale(const JobDev& jd, float adapt, int k, float cool) {
    const int RL = rungs_per_ladder(jd), pos = k % RL;
    return adapt * (RL > 1 ? 0.15f + 1.85f * (float)pos / (float)(RL - 1) : 1.f) * sqrtf(cool);
}

// Container side of rung k when the job's side is B: B itself, or under
// SQS_JOB_TARGETS the reference's target below the best,
// max(sqrt n + 1e-6, B (1 - shrink m(pos))) (seeded.cu:478-481, with the
// shrink relative to the side).
__device__ __forceinline__ float rung_side(const JobDev& jd, float B, int k) {
    if (!(jd.flags & kTargets)) return B;
    const int RL = rungs_per_ladder(jd);
    const float lb = sqrtf((float)jd.n) + 1e-6f;
    return fmaxf(lb, B * (1.f - jd.shrink * target_mult(k % RL, RL)));
}

struct CtaShared {
    JobDev jd;
    JobMut jm;
    float temps[kMaxR];
    long long wE[kMaxRl];      // this CTA's replica energies at a checkpoint
    double wL[kMaxRl];         // this CTA's candidate certified sides at a checkpoint
    double wlam[kMaxRl], wx0[kMaxRl], wy0[kMaxRl];
    float wside[kMaxRl];       // each replica's container side (per rung under SQS_JOB_TARGETS)
    int wbad[kMaxRl];          // cell-list overflow per warp
    int decision_win;          // global replica index of the new best (-1: none)
    int bad;                   // any overflow in the cluster
    int reset0;                // SQS_JOB_TARGETS: the gain resets every rung of ladder 0, not only heads
    float newL;
    unsigned long long props[kMaxRl], accs[kMaxRl];
    long long red[3 * kMaxRl];   // group sums: up to three values a warp
    long long qE;              // energy of the replica quenched by this CTA
    long long qEv[kMaxRl];     // each replica's energy through a group quench
};

// MOVES: whether the move-set options (adaptation, collective moves, kicks)
// are compiled in; jobs without them run the leaner instance.
template <int V>
struct IntTag {
    static constexpr int value = V;
};

// A proposal's move: the square (-1: nothing moved) and its old and new
// cells, one byte per coordinate (grids are at most 64 / 1.59 < 256 wide).
struct Moved {
    int i, cells;
};
__device__ __forceinline__ int pack_cells(int ox, int oy, int nx, int ny) {
    return ox | (oy << 8) | (nx << 16) | (ny << 24);
}
// Did move (mi, mc) change what a proposal of square ik from cells ck read?
__device__ __forceinline__ bool touches(int mi, int mc, int ik, int ck) {
    if (mi < 0) return false;
    const int bx = ck & 0xff, by = (ck >> 8) & 0xff;
    const int ox = mc & 0xff, oy = (mc >> 8) & 0xff, nx = (mc >> 16) & 0xff, ny = (int)((unsigned)mc >> 24);
    return mi == ik || (abs(ox - bx) <= 1 && abs(oy - by) <= 1) || (abs(nx - bx) <= 1 && abs(ny - by) <= 1);
}

template <bool MOVES>
__global__ void __launch_bounds__(32 * kMaxRl) anneal_kernel(const int32_t* __restrict__ job_list,
                                                      const JobDev* __restrict__ jdev, JobMut* __restrict__ jmut,
                                                      float4* __restrict__ pos, double* __restrict__ best,
                                                      int slice_sweeps, int dyn_bytes) {
    cg::cluster_group cluster = cg::this_cluster();
    __shared__ CtaShared S;
    extern __shared__ __align__(16) unsigned char dyn[];
    const int rank = (int)cluster.block_rank();
    const int job = job_list[blockIdx.x / cluster.num_blocks()];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    if (tid == 0) {
        S.jd = jdev[job];
        S.jm = jmut[job];
    }
    __syncthreads();
    const JobDev& jd = S.jd;
    if (S.jm.status != kRunning) return;  // identical in every CTA of the cluster
    const int n = jd.n, R = jd.R, Rl = jd.Rl;
    const int r = rank * Rl + w;  // global replica index of this warp
    const bool active = w < Rl;
    if (tid < R) S.temps[tid] = rung_temp(jd, tid);
    const int64_t rb = replica_smem_bytes(n, jd.Gmax);
    Rep rep = rep_view(dyn + (active ? w : 0) * rb, n, jd.Gmax);
    float L = S.jm.L;  // the job's side: every replica's, or under SQS_JOB_TARGETS the best the rung sides hang from
    Grid g = make_grid(L, jd.Gmax, jd.cell);
    // this replica's side (walls, move clamps, kicks, quench)
    float Lr = active ? rung_side(jd, L, S.jm.perm[r]) : L;
    if (active && lane == 0) S.wside[w] = Lr;
    const uint32_t k0 = (uint32_t)jd.seed, k1 = (uint32_t)(jd.seed >> 32);

    // load the replica
    if (active) {
        const float4* src = pos + jd.pos_off + (int64_t)r * n;
        for (int i = lane; i < n; i += 32) {
            const float4 p = src[i];
            float s, c;
            state_trig(p.z, &s, &c);
            rep.sq[i] = make_float4(p.x, p.y, c, s);
            rep.ang[i] = p.z;
        }
        __syncwarp();
        const bool ok = build_cells(rep, n, g, lane);
        if (lane == 0) S.wbad[w] = !ok;
    }
    __syncthreads();
    cluster.sync();
    if (tid == 0) {
        int bad = 0;
        for (int q = 0; q < (int)cluster.num_blocks(); ++q) {
            const CtaShared* o = cluster.map_shared_rank(&S, q);
            for (int k = 0; k < Rl; ++k) bad |= o->wbad[k];
        }
        S.bad = bad;
    }
    cluster.sync();
    if (S.bad) {
        if (rank == 0 && tid == 0) jmut[job].status = kErrCells;
        return;
    }
    long long E = 0;
    if (active) {
        E = S.jm.done == 0 ? full_energy(rep, n, g, Lr, lane) : S.jm.E[r];
    }
    unsigned long long props = 0, accs = 0;
    int ovf = 0;
    // move-set options: step adaptation with a cooling cycle of 200 exchange
    // rounds (temperatures x 0.002^(k/199), steps x its square root)
    const bool adaptive = MOVES && (jd.flags & kMoveAdapt) != 0;
    float adapt = (MOVES && active) ? S.jm.adapt[r] : 1.f;
    int win = (MOVES && active) ? S.jm.win[r] : 0;
    float cool = cool_of(adaptive, S.jm.xround);
    float invT = active ? 1.0f / (S.temps[S.jm.perm[r]] * cool) : 0.f;
    float4* save = pos + jd.pos_off + (int64_t)r * n;  // this replica's HBM slot: free while the slice runs

    // Proposals are numbered per replica across the whole job (a sweep is n
    // of them); checkpoints fall after every xprops proposals and at the end
    // of the budget; a slice ends after its sweeps' worth of proposals.
    const int64_t P_total = jd.props_total, xp = jd.xprops;
    int64_t p_at = S.jm.done;
    const int64_t p_end = min(P_total, p_at + (int64_t)(jd.slice > 0 ? jd.slice : slice_sweeps) * n);
    while (p_at < p_end) {
        const int64_t next_cp = min(P_total, (p_at / xp + 1) * xp);
        const int64_t stop = min(next_cp, p_end);
        if (active) {
            for (int64_t base = p_at; base < stop; base += 32) {
                // Lane l draws proposal base + l: two Philox blocks keyed by
                // (proposal index, replica, 0 / 1), Box-Muller for the centre
                // step and the angle step, the uniform of the Metropolis test.
                // Each proposal then broadcasts its draws.
                const int kn = (int)(stop - base < 32 ? stop - base : 32);
                int di = 0;
                float ddx = 0.f, ddy = 0.f, dda = 0.f, du = 0.f;
                if (lane < kn) {
                    const uint64_t ev = (uint64_t)(base + lane);
                    const U4 ra = philox4x32_10(U4{(uint32_t)ev, (uint32_t)(ev >> 32), (uint32_t)r, 0u}, k0, k1);
                    const U4 rb = philox4x32_10(U4{(uint32_t)ev, (uint32_t)(ev >> 32), (uint32_t)r, 1u}, k0, k1);
                    di = (int)(((uint64_t)ra.x * (uint64_t)n) >> 32);
                    if (adaptive) {
                        // the reference search's steps: uniform in +-sigma
                        // for each coordinate and the angle (seeded.cu:508-510)
                        ddx = jd.sigma_xy * (2.f * u01(ra.y) - 1.f);
                        ddy = jd.sigma_xy * (2.f * u01(ra.z) - 1.f);
                        dda = jd.sigma_a * (2.f * u01(ra.w) - 1.f);
                    } else {
                        const float rad1 = sqrtf(-2.f * __logf(u01(ra.y)));
                        float sn1, cs1;
                        __sincosf(6.2831853f * u01(ra.z), &sn1, &cs1);
                        const float rad2 = sqrtf(-2.f * __logf(u01(ra.w)));
                        const float n2 = rad2 * __cosf(6.2831853f * u01(rb.x));
                        ddx = jd.sigma_xy * rad1 * cs1;
                        ddy = jd.sigma_xy * rad1 * sn1;
                        dda = jd.sigma_a * n2;
                    }
                    du = u01(rb.y);
                    if (MOVES && (jd.flags & kMoveCollective)) di |= (int)(rb.z % 7u) << 16;  // move mode
                }
                // one lane moves square i to its new state and cell
                auto apply_move = [&](int i, float nx, float ny, float nc, float ns, float na, int oc, int ncell) {
                    rep.sq[i] = make_float4(nx, ny, nc, ns);
                    rep.ang[i] = na;
                    if (oc != ncell) {
                        const int m = rep.cnt[oc];
                        for (int t = 0; t < m; ++t) {
                            if (rep.slot[oc * kCellK + t] == (uint16_t)i) {
                                rep.slot[oc * kCellK + t] = rep.slot[oc * kCellK + m - 1];
                                break;
                            }
                        }
                        rep.cnt[oc] = (uint8_t)(m - 1);
                        rep.slot[ncell * kCellK + rep.cnt[ncell]] = (uint16_t)i;
                        rep.cnt[ncell] = (uint8_t)(rep.cnt[ncell] + 1);
                    }
                };
                // proposal q of this batch, evaluated by the whole warp; returns
                // the square it moved (-1: none) and its old and new cells
                auto single = [&](int q) -> Moved {
                    Moved mv{-1, 0};
                    const int dpk = __shfl_sync(0xffffffffu, di, q);
                    const int i = dpk & 0xffff, mode = dpk >> 16;
                    const float sdx = __shfl_sync(0xffffffffu, ddx, q), sdy = __shfl_sync(0xffffffffu, ddy, q);
                    const float sda = __shfl_sync(0xffffffffu, dda, q), u_acc = __shfl_sync(0xffffffffu, du, q);
                    float sc = 1.f;  // step scale (adaptive moves)
                    const uint64_t pidx = (uint64_t)(base + q);
                    if (adaptive) {
                        sc = step_scale(jd, adapt, S.jm.perm[r], cool);
                        if ((pidx & 15u) == 0) sc *= 3.5f;
                    }
                    const float dx = fminf(kMaxStep, fmaxf(-kMaxStep, sdx * sc));
                    const float dy = fminf(kMaxStep, fmaxf(-kMaxStep, sdy * sc));
                    const float da = sda * sc;
                    bool acc;
                    if (MOVES && mode != 0) {
                        acc = collective_move(rep, g, n, Lr, lane, mode, i, dx, dy, da, u_acc, invT, E, save, &ovf);
                        ++props;
                        accs += acc;
                    } else {
                    const float4 P = rep.sq[i];
                    // keep centres in [0.5, Lr - 0.5] without ever moving a square
                    // further than the clamped step (it may start outside)
                    const float nx = fminf(fmaxf(P.x, Lr - 0.5f), fmaxf(fminf(P.x, 0.5f), P.x + dx));
                    const float ny = fminf(fmaxf(P.y, Lr - 0.5f), fmaxf(fminf(P.y, 0.5f), P.y + dy));
                    float na = rep.ang[i] + da;
                    na = na - kHalfPiF * floorf(na * (1.0f / kHalfPiF));
                    if (!(na >= 0.f && na < kHalfPiF)) na = 0.f;
                    float ns, nc;
                    state_trig(na, &ns, &nc);
                    const int ocx = g.cx(P.x), ocy = g.cx(P.y);
                    long long dq = 0;
                    if (lane == 0) dq = qe(wall_e(nx, ny, nc, ns, Lr)) - qe(wall_e(P.x, P.y, P.z, P.w, Lr));
                    for_block(rep, g, ocx, ocy, lane, [&](int j) {
                        const long long d = pair_delta(rep.sq[j], nx, ny, nc, ns, P);
                        dq += j != i ? d : 0;
                    });
                    dq = warp_sum_dq(dq);
                    const float de = (float)dq * (1.0f / kEScale);
                    acc = dq <= 0 || u_acc < __expf(-de * invT);
                    const int ncx = g.cx(nx), ncy = g.cx(ny);
                    const int oc = ocy * g.G + ocx, ncell = ncy * g.G + ncx;
                    if (acc && oc != ncell && rep.cnt[ncell] >= kCellK) {
                        acc = false;
                        ++ovf;
                    }
                    ++props;
                    if (acc) {
                        ++accs;
                        E += dq;
                        if (lane == 0) apply_move(i, nx, ny, nc, ns, na, oc, ncell);
                        mv = Moved{i, pack_cells(ocx, ocy, ncx, ncy)};
                    }
                    }
                    if (adaptive) {  // every 16 proposals: steer toward 25% acceptance
                        win += acc;
                        if (((pidx + 1u) & 15u) == 0) {
                            adapt = fmaxf(0.1f, fminf(4.0f, adapt * expf(((float)win / 16.f - 0.25f) * 0.5f)));
                            win = 0;
                        }
                    }
                    __syncwarp();
                    return mv;
                };
                // Proposals q .. q + M - 1 evaluated at once, one per group of
                // 32 / M lanes, all against the current state, then decided in
                // order.  A proposal's result stands unless an earlier move of
                // the group that was accepted touched what it read: the same
                // square, or an old or new cell of that move inside its 3x3
                // block (cells are wider than a step, so a move changes a
                // square's cell by at most one; every other read -- counts and
                // slots of the block, squares in it, the count of its target
                // cell -- lies in that block).  Then the whole warp evaluates it
                // again on the current state.  Energies are exact and
                // order-free, so the trajectory is the one-at-a-time trajectory,
                // bit for bit.
                auto group = [&](int q, auto mtag) {
                    constexpr int M = decltype(mtag)::value, W = 32 / M;
                    const int grp = lane / W, gl = lane % W;
                    const int qs = q + grp;
                    const int i = __shfl_sync(0xffffffffu, di, qs) & 0xffff;
                    const float sdx = __shfl_sync(0xffffffffu, ddx, qs), sdy = __shfl_sync(0xffffffffu, ddy, qs);
                    const float sda = __shfl_sync(0xffffffffu, dda, qs), u_acc = __shfl_sync(0xffffffffu, du, qs);
                    const float dx = fminf(kMaxStep, fmaxf(-kMaxStep, sdx));
                    const float dy = fminf(kMaxStep, fmaxf(-kMaxStep, sdy));
                    const float4 P = rep.sq[i];
                    const float nx = fminf(fmaxf(P.x, Lr - 0.5f), fmaxf(fminf(P.x, 0.5f), P.x + dx));
                    const float ny = fminf(fmaxf(P.y, Lr - 0.5f), fmaxf(fminf(P.y, 0.5f), P.y + dy));
                    float na = rep.ang[i] + sda;
                    na = na - kHalfPiF * floorf(na * (1.0f / kHalfPiF));
                    if (!(na >= 0.f && na < kHalfPiF)) na = 0.f;
                    float ns, nc;
                    state_trig(na, &ns, &nc);
                    const int ocx = g.cx(P.x), ocy = g.cx(P.y);
                    long long dq = 0;
                    if (gl == 0) dq = qe(wall_e(nx, ny, nc, ns, Lr)) - qe(wall_e(P.x, P.y, P.z, P.w, Lr));
                    for_block<W>(rep, g, ocx, ocy, gl, [&](int j) {
                        const long long d = pair_delta(rep.sq[j], nx, ny, nc, ns, P);
                        dq += j != i ? d : 0;
                    });
                    // exact sum over the group's lanes: hi * 2^20 + lo parts
                    // (a lane's term is below 2^46, so both parts stay in 32 bits)
                    int hi = (int)(dq >> 20);
                    unsigned lo = (unsigned)(dq & 0xFFFFF);
#pragma unroll
                    for (int off = W / 2; off > 0; off >>= 1) {
                        hi += __shfl_xor_sync(0xffffffffu, hi, off);
                        lo += __shfl_xor_sync(0xffffffffu, lo, off);
                    }
                    const long long mine = (long long)hi * 1048576ll + (long long)lo;
                    const float de = (float)mine * (1.0f / kEScale);
                    const int ncx = g.cx(nx), ncy = g.cx(ny);
                    const int oc = ocy * g.G + ocx, ncell = ncy * g.G + ncx;
                    int acc = mine <= 0 || u_acc < __expf(-de * invT);
                    int ov = 0;
                    if (acc && oc != ncell && rep.cnt[ncell] >= kCellK) {
                        acc = 0;
                        ov = 1;
                    }
                    const int cells = pack_cells(ocx, ocy, ncx, ncy);
                    int mi[M], mc[M];  // the group's moves so far: square (-1: none), cells
#pragma unroll
                    for (int k = 0; k < M; ++k) {
                        const int src = k * W;
                        const int ik = __shfl_sync(0xffffffffu, i, src), ck = __shfl_sync(0xffffffffu, cells, src);
                        bool redo = false;
#pragma unroll
                        for (int m = 0; m < k; ++m) redo |= touches(mi[m], mc[m], ik, ck);
                        if (redo) {
                            const Moved mv = single(q + k);
                            mi[k] = mv.i;
                            mc[k] = mv.cells;
                        } else {
                            const int ak = __shfl_sync(0xffffffffu, acc, src), ovk = __shfl_sync(0xffffffffu, ov, src);
                            const unsigned dlo = __shfl_sync(0xffffffffu, (unsigned)(unsigned long long)mine, src);
                            const int dhi = __shfl_sync(0xffffffffu, (int)(mine >> 32), src);
                            ++props;
                            accs += ak;
                            ovf += ovk;
                            if (ak) E += (long long)(((unsigned long long)(unsigned)dhi << 32) | dlo);
                            if (ak && lane == src) apply_move(i, nx, ny, nc, ns, na, oc, ncell);
                            __syncwarp();
                            mi[k] = ak ? ik : -1;
                            mc[k] = ck;
                        }
                    }
                };
                // groups need room: on small grids most proposals would be
                // evaluated twice; the move-set instance keeps one at a time
                // (its step scale follows the acceptance of the previous move)
                const bool fours = !MOVES && g.G >= 8, twos = !MOVES && g.G >= 4;
                for (int q = 0; q < kn;) {
                    if (fours && q + 3 < kn) {
                        group(q, IntTag<4>{});
                        q += 4;
                    } else if (twos && q + 1 < kn) {
                        group(q, IntTag<2>{});
                        q += 2;
                    } else {
                        single(q);
                        ++q;
                    }
                }
            }
        }
        p_at = stop;
        // ---- checkpoint: best-state search, shrink, replica exchange.  Only
        // after every xprops proposals (and at the end of the budget), so a
        // job's trajectory does not depend on how it is sliced.
        if (p_at != next_cp) break;  // the slice ends between checkpoints
        const bool xpoint = p_at % xp == 0;
        if (MOVES && (jd.flags & kMoveQuenchAll) && jd.quench_iters > 0) {
            // every replica at once, each by its own group of gw warps (the
            // launch gives each replica gw = blockDim / (32 Rl) warps); the
            // scratch (kQuenchScr n float4 a replica) in shared memory after
            // the replicas when the launch left room for all of them, else
            // the replica's own block of the job's scratch in HBM
            const int gw = (int)(blockDim.x >> 5) / Rl, q = w / gw;
            const bool smem_scr = (int64_t)dyn_bytes >= (int64_t)Rl * (rb + (int64_t)sizeof(float4) * kQuenchScr * n);
            float4* qw = smem_scr ? reinterpret_cast<float4*>(dyn + (int64_t)Rl * rb) + (int64_t)q * kQuenchScr * n
                                  : pos + jd.scr_off + ((int64_t)rank * Rl + q) * kQuenchScr * n;
            if (gw == 1) {
                if (active) E = quench_grp(WarpGrp{lane}, rep, n, g, Lr, jd.quench_iters, jd.quench_stall, qw, E);
            } else {
                if (active && lane == 0) S.qEv[w] = E;
                __syncthreads();
                if (q < Rl) {
                    const BarGrp gp{1 + q, gw, q * gw * 32, S.red + 3 * q * gw};
                    const Rep cr = rep_view(dyn + q * rb, n, jd.Gmax);
                    const long long e =
                        quench_grp(gp, cr, n, g, S.wside[q], jd.quench_iters, jd.quench_stall, qw, S.qEv[q]);
                    if (gp.t() == 0) S.qEv[q] = e;
                }
                __syncthreads();
                if (active) E = S.qEv[w];
            }
            __syncthreads();
        } else {
            // the replica on the coldest rung, by every thread of the CTA that
            // holds it; its scratch in shared memory after the replicas when
            // the launch left room, else this CTA's block of the job's scratch
            float4* qs = (int64_t)dyn_bytes >= (int64_t)Rl * rb + (int64_t)sizeof(float4) * kQuenchScr * n
                             ? reinterpret_cast<float4*>(dyn + (int64_t)Rl * rb)
                             : pos + jd.scr_off + (int64_t)rank * kQuenchScr * n;
            int cold = 0;
            for (int q = 0; q < R; ++q)
                if (S.jm.perm[q] == 0) cold = q;
            if (jd.quench_iters > 0 && cold / Rl == rank) {
                if (w == cold % Rl && lane == 0) S.qE = E;
                __syncthreads();
                const Rep cr = rep_view(dyn + (cold % Rl) * rb, n, jd.Gmax);
                const long long qe_out = quench_grp(CtaGrp{S.red}, cr, n, g, S.wside[cold % Rl], jd.quench_iters,
                                                    jd.quench_stall, qs, S.qE);
                if (w == cold % Rl) E = qe_out;
                __syncthreads();
            }
        }
        if (active) {
            double Lc = 1e30, lam = 0, x0 = 0, y0 = 0;
            // any state whose overlaps a dilation of at most 0.8% removes is a
            // certified candidate (penetrations of depth d cost about d^2 each,
            // so the energy gate skips states that cannot pass); under
            // SQS_JOB_CERT_ALL every replica is measured, as the reference
            // search measures every chain after its polish (seeded.cu:716)
            if (E < qe(1e-4f) || (jd.flags & kCertAll)) Lc = cert_side(rep, n, g, lane, lam, x0, y0);
            if (lane == 0) {
                S.wE[w] = E;
                S.wL[w] = Lc;
                S.wlam[w] = lam;
                S.wx0[w] = x0;
                S.wy0[w] = y0;
            }
        }
        __syncthreads();
        cluster.sync();
        if (tid == 0) {
            // every CTA takes the same decisions from the same gathered values
            long long Eall[kMaxR];
            // under SQS_JOB_TARGETS only a side below the initial one counts, as
            // the reference's chain bests start at the seed's side (seeded.cu:883)
            const double best0 = (jd.flags & kTargets) ? fmin(S.jm.best_L, (double)jd.L0) : S.jm.best_L;
            double bestc = best0;
            int win = -1;
            for (int q = 0; q < (int)cluster.num_blocks(); ++q) {
                const CtaShared* o = cluster.map_shared_rank(&S, q);
                for (int k = 0; k < Rl; ++k) {
                    Eall[q * Rl + k] = o->wE[k];
                    if (o->wL[k] < bestc) {
                        bestc = o->wL[k];
                        win = q * Rl + k;
                    }
                }
            }
            S.decision_win = win;
            S.newL = L;
            S.reset0 = 0;
            const bool targets = (jd.flags & kTargets) != 0;
            if (win >= 0) {
                const double gain = best0 < 1e29 ? best0 - bestc : 0.0;
                S.jm.best_L = bestc;
                S.jm.improvements += 1;
                const float lb = sqrtf((float)n) + 1e-6f;
                // the job's side: the new best (the rung targets hang below it), or
                // the best shrunk by the job's factor
                float nl = targets ? (float)fmin((double)L, bestc)
                                   : (float)(fmin((double)L, bestc) * (1.0 - (double)jd.shrink));
                if (nl < lb) nl = lb;
                if (nl < L) {
                    S.newL = nl;
                    S.jm.shrinks += 1;
                }
                // a large gain resets every rung of ladder 0 to the new best (seeded.cu:929)
                S.reset0 = targets && gain > 5e-4;
            }
            // replica exchange between neighbouring rungs of each ladder, alternating
            // parity; under SQS_JOB_TARGETS only in rounds without a new best, as the
            // reference swaps only in epochs that did not improve (seeded.cu:939-941)
            if (xpoint && !(targets && win >= 0)) {
                int holder[kMaxR];
                for (int q = 0; q < R; ++q) holder[S.jm.perm[q]] = q;
                const int par = S.jm.xround & 1;
                const int RL = rungs_per_ladder(jd);
                for (int k = 0; k + 1 < R; ++k) {
                    const int pos = k % RL;
                    if ((pos & 1) != par || pos + 1 >= RL) continue;
                    const int a = holder[k], b = holder[k + 1];
                    const U4 u = philox4x32_10(U4{(uint32_t)S.jm.xround, (uint32_t)k, 0u, 0x7fffffffu}, k0, k1);
                    const float d = (1.0f / S.temps[k] - 1.0f / S.temps[k + 1]) *
                                    ((float)(Eall[a] - Eall[b]) * (1.0f / kEScale)) / cool;
                    S.jm.xatt += 1;
                    if (d >= 0.f || u01(u.x) < expf(d)) {
                        S.jm.xacc += 1;
                        S.jm.perm[a] = k + 1;
                        S.jm.perm[b] = k;
                        holder[k] = b;
                        holder[k + 1] = a;
                    }
                }
            }
            if (xpoint) S.jm.xround += 1;
        }
        cluster.sync();
        __syncthreads();
        if (adaptive) cool = cool_of(true, S.jm.xround);
        const bool targets = MOVES && (jd.flags & kTargets) != 0;
        if (active) {
            invT = 1.0f / (S.temps[S.jm.perm[r]] * cool);
            if (S.decision_win == r) {
                // new best: dilated, translated to the origin, angles in [0, pi/2)
                double* dst = best + jd.best_off;
                const double lam = S.wlam[w], x0 = S.wx0[w], y0 = S.wy0[w];
                for (int i = lane; i < n; i += 32) {
                    dst[3 * i] = __dsub_rn(__dmul_rn((double)rep.sq[i].x, lam), x0);
                    dst[3 * i + 1] = __dsub_rn(__dmul_rn((double)rep.sq[i].y, lam), y0);
                    dst[3 * i + 2] = (double)rep.ang[i];
                }
            }
        }
        if (targets && S.decision_win >= 0) {  // the new best is read by the ladder heads below
            __threadfence();
            __syncthreads();
            cluster.sync();
        }
        const bool regrid = S.newL < L;
        if (regrid || targets) {
            const float f = S.newL / L;
            if (regrid) {
                L = S.newL;
                g = make_grid(L, jd.Gmax, jd.cell);
            }
            if (active) {
                const int rung = S.jm.perm[r];
                const float Ln = rung_side(jd, L, rung);
                const int RL = rungs_per_ladder(jd);
                const bool reset = targets && S.decision_win >= 0 && (rung % RL == 0 || (S.reset0 && rung < RL));
                if (reset) {
                    // ladder head: the new best, scaled into its own side (seeded.cu:928-936)
                    const double* src = best + jd.best_off;
                    const double sc = (double)Ln / (double)L;
                    for (int i = lane; i < n; i += 32) {
                        const float a = (float)src[3 * i + 2];
                        float sn, cs;
                        state_trig(a, &sn, &cs);
                        rep.sq[i] = make_float4((float)(src[3 * i] * sc), (float)(src[3 * i + 1] * sc), cs, sn);
                        rep.ang[i] = a;
                    }
                } else if (regrid && !targets) {
                    for (int i = lane; i < n; i += 32) {
                        rep.sq[i].x *= f;
                        rep.sq[i].y *= f;
                    }
                }
                __syncwarp();
                if (reset || regrid) {
                    const bool ok = build_cells(rep, n, g, lane);
                    if (lane == 0) S.wbad[w] = !ok;
                }
                const bool changed = reset || regrid || Ln != Lr;
                Lr = Ln;
                if (lane == 0) S.wside[w] = Lr;
                if (changed) E = full_energy(rep, n, g, Lr, lane);
            }
            if (regrid || (targets && S.decision_win >= 0)) {
                __syncthreads();
                cluster.sync();
                if (tid == 0) {
                    int bad = 0;
                    for (int q = 0; q < (int)cluster.num_blocks(); ++q) {
                        const CtaShared* o = cluster.map_shared_rank(&S, q);
                        for (int k = 0; k < Rl; ++k) bad |= o->wbad[k];
                    }
                    S.bad = bad;
                }
                cluster.sync();
                if (S.bad) {
                    if (rank == 0 && tid == 0) jmut[job].status = kErrCells;
                    return;
                }
            }
            __syncthreads();
        }
        // overlapped replicas are kicked (the round just completed decides
        // whether the worst square is also moved)
        if (MOVES && active && (jd.flags & kMoveKick) && E > qe(1e-12f))
            E = kick_replica(rep, g, n, Lr, lane, r, S.jm.xround, k0, k1, E, save);
    }

    // ---- write the slice back
    if (active) {
        float4* dst = pos + jd.pos_off + (int64_t)r * n;
        for (int i = lane; i < n; i += 32) dst[i] = make_float4(rep.sq[i].x, rep.sq[i].y, rep.ang[i], 0.f);
        if (lane == 0) {
            jmut[job].E[r] = E;
            if (MOVES) {
                jmut[job].adapt[r] = adapt;
                jmut[job].win[r] = win;
            }
            atomicAdd(reinterpret_cast<unsigned long long*>(&jmut[job].proposals), props);
            atomicAdd(reinterpret_cast<unsigned long long*>(&jmut[job].accepted), accs);
            if (ovf) atomicAdd(&jmut[job].overflows, ovf);
        }
    }
    if (rank == 0 && tid == 0) {
        JobMut& m = jmut[job];
        m.L = L;
        m.done = p_end;
        m.xround = S.jm.xround;
        m.status = p_end >= P_total ? kFinished : kRunning;
        m.shrinks = S.jm.shrinks;
        m.improvements = S.jm.improvements;
        m.best_L = S.jm.best_L;
        m.xatt = S.jm.xatt;
        m.xacc = S.jm.xacc;
        for (int q = 0; q < R; ++q) m.perm[q] = S.jm.perm[q];
    }
}

// Final state of every replica, read back by sqs_anneal_batch_trace: one
// warp per (job, replica) loads the replica as the annealer left it, rebuilds
// its cell list on the job's grid and recomputes, with the annealer's own
// device functions, its fixed-point energy from scratch (equal, bit for bit,
// to the running energy the proposals kept when nothing drifts) and its FP64
// dilation-certified side, and reports the temperature and step scale its
// next proposal would use.
__global__ void __launch_bounds__(32) trace_kernel(const int2* __restrict__ items, const JobDev* __restrict__ jdev,
                                                   const JobMut* __restrict__ jmut, const float4* __restrict__ pos,
                                                   TraceRec* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char dyn[];
    const int2 it = items[blockIdx.x];
    const JobDev& jd = jdev[it.x];
    const JobMut& jm = jmut[it.x];
    const int n = jd.n, r = it.y, lane = threadIdx.x;
    const Rep rep = rep_view(dyn, n, jd.Gmax);
    const Grid g = make_grid(jm.L, jd.Gmax, jd.cell);
    const float L = rung_side(jd, jm.L, jm.perm[r]);
    const float4* src = pos + jd.pos_off + (int64_t)r * n;
    for (int i = lane; i < n; i += 32) {
        const float4 p = src[i];
        float sn, cs;
        state_trig(p.z, &sn, &cs);
        rep.sq[i] = make_float4(p.x, p.y, cs, sn);
        rep.ang[i] = p.z;
    }
    __syncwarp();
    const bool ok = build_cells(rep, n, g, lane);
    const long long E = full_energy(rep, n, g, L, lane);
    double lam = 0, x0 = 0, y0 = 0;
    const double Lc = cert_side(rep, n, g, lane, lam, x0, y0);
    if (lane == 0) {
        const bool adaptive = (jd.flags & kMoveAdapt) != 0;
        const float cool = cool_of(adaptive, jm.xround);
        const int rung = jm.perm[r];
        TraceRec t;
        t.E_full = E;
        t.L_cert = Lc;
        t.lam = lam;
        t.temp = rung_temp(jd, rung) * cool;
        t.step = adaptive ? step_scale(jd, jm.adapt[r], rung, cool) : 1.f;
        t.side = L;
        t.rung = rung;
        t.cells_ok = ok ? 1 : 0;
        t.pad = 0;
        out[blockIdx.x] = t;
    }
}

int launch_trace(cudaStream_t stream, int items, const int2* list, const JobDev* jdev, const JobMut* jmut,
                 const float4* pos, TraceRec* out, size_t smem) {
    static bool attr_done[64] = {false};
    int dev = 0;
    SQS_CUDA(cudaGetDevice(&dev));
    if (!attr_done[dev & 63]) {
        SQS_CUDA(cudaFuncSetAttribute(trace_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kAnnealSmemLimit));
        attr_done[dev & 63] = true;
    }
    if (items <= 0) return SQS_OK;
    trace_kernel<<<items, 32, smem, stream>>>(list, jdev, jmut, pos, out);
    SQS_CUDA(cudaGetLastError());
    return SQS_OK;
}

// Kernel attributes (dynamic shared memory up to the opt-in limit,
// non-portable cluster sizes), once per device; call before any capture.
int prime_anneal() {
    static bool attr_done[64] = {false};
    int dev = 0;
    SQS_CUDA(cudaGetDevice(&dev));
    if (!attr_done[dev & 63]) {
        for (int v = 0; v < 2; ++v) {
            const void* fn = v ? (const void*)anneal_kernel<true> : (const void*)anneal_kernel<false>;
            cudaFuncAttributes fa;
            SQS_CUDA(cudaFuncGetAttributes(&fa, fn));
            SQS_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          232448 - (int)fa.sharedSizeBytes));
            SQS_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        }
        attr_done[dev & 63] = true;
    }
    return SQS_OK;
}

static cudaLaunchConfig_t anneal_config(int clusters, int cs, int Rl, size_t smem, cudaStream_t stream,
                                        cudaLaunchAttribute* attr, int gw = 1) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(clusters * cs), 1, 1);
    cfg.blockDim = dim3((unsigned)(Rl * 32 * gw), 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

// Clusters of this shape (gw warps a replica) that can be resident at once
// (one wave), memoized per device and shape.
static int max_clusters_gw(int cs, int Rl, size_t smem, bool moves, int gw, int* out) {
    static std::mutex mu;
    static std::map<std::tuple<int, int, int, size_t, bool, int>, int> memo;
    int dev = 0;
    SQS_CUDA(cudaGetDevice(&dev));
    const auto key = std::make_tuple(dev, cs, Rl, smem, moves, gw);
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = memo.find(key);
        if (it != memo.end()) {
            *out = it->second;
            return SQS_OK;
        }
    }
    if (int r = prime_anneal()) return r;
    cudaLaunchAttribute attr[1];
    const cudaLaunchConfig_t cfg = anneal_config(1, cs, Rl, smem, nullptr, attr, gw);
    int num = 0;
    if (moves) SQS_CUDA(cudaOccupancyMaxActiveClusters(&num, anneal_kernel<true>, &cfg));
    else SQS_CUDA(cudaOccupancyMaxActiveClusters(&num, anneal_kernel<false>, &cfg));
    std::lock_guard<std::mutex> lk(mu);
    memo[key] = num;
    *out = num;
    return SQS_OK;
}

int anneal_max_clusters(int cs, int Rl, size_t smem, bool moves, int* out) {
    return max_clusters_gw(cs, Rl, smem, moves, 1, out);
}

// Warps a replica for a launch of njobs clusters: 1 (the replica's own warp),
// or with the move-set options the most, up to kMaxRl / Rl, that keep as
// many of the launch's clusters resident at once.  The extra warps idle
// while their CTA anneals and join the checkpoint quench, which
// SQS_JOB_QUENCH_ALL runs for every replica at once (same results: the
// quench's sums are integers).
static int quench_warps(int njobs, int cs, int Rl, size_t smem, bool moves) {
    if (!moves || Rl >= kMaxRl) return 1;
    int base = 0;
    if (max_clusters_gw(cs, Rl, smem, moves, 1, &base) != SQS_OK) return 1;
    const int need = std::min(njobs, base);
    for (int gw = kMaxRl / Rl; gw > 1; gw /= 2) {
        int m = 0;
        if (max_clusters_gw(cs, Rl, smem, moves, gw, &m) == SQS_OK && m >= need) return gw;
    }
    return 1;
}

int launch_anneal(cudaStream_t stream, int njobs, int cs, int Rl, size_t smem, bool moves, const int32_t* job_list,
                  const JobDev* jdev, JobMut* jmut, float4* pos, double* best, int slice) {
    if (int r = prime_anneal()) return r;
    cudaLaunchAttribute attr[1];
    const int gw = quench_warps(njobs, cs, Rl, smem, moves);
    const cudaLaunchConfig_t cfg = anneal_config(njobs, cs, Rl, smem, stream, attr, gw);
    if (moves) SQS_CUDA(cudaLaunchKernelEx(&cfg, anneal_kernel<true>, job_list, jdev, jmut, pos, best, slice, (int)smem));
    else SQS_CUDA(cudaLaunchKernelEx(&cfg, anneal_kernel<false>, job_list, jdev, jmut, pos, best, slice, (int)smem));
    return SQS_OK;
}

// Shared memory of a launch whose largest job needs rb bytes a replica and
// has n_max squares: the replicas, plus room for the checkpoint quench's
// scratch (kQuenchScr n float4 per quench) when that fits and keeps as many
// clusters resident -- the quench then runs on shared instead of global
// memory (same results).  Launches with the move-set options first try room
// for every replica's quench (SQS_JOB_QUENCH_ALL quenches them all at once),
// then for one.  `need` is how many clusters the launch must keep resident:
// a size is taken when it keeps min(need, the clusters the bare replicas
// allow) resident, so a launch of a few jobs always gets the room.
size_t anneal_smem(int cs, int Rl, int64_t rb, int n_max, bool moves, int need) {
    const size_t base = (size_t)(rb * Rl), q1 = sizeof(float4) * kQuenchScr * (size_t)n_max;
    const size_t one = base + q1, all = moves ? base + q1 * (size_t)Rl : one;
    static std::mutex mu;
    static std::map<std::tuple<int, int, int, size_t, size_t, bool, int>, size_t> memo;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return base;
    const auto key = std::make_tuple(dev, cs, Rl, base, all, moves, need);
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = memo.find(key);
        if (it != memo.end()) return it->second;
    }
    int a = 0;
    size_t pick = base;
    if (anneal_max_clusters(cs, Rl, base, moves, &a) == SQS_OK) {
        for (const size_t cand : {all, one}) {
            int b = 0;
            if (cand <= kAnnealSmemLimit && anneal_max_clusters(cs, Rl, cand, moves, &b) == SQS_OK &&
                b >= std::min(need, a)) {
                pick = cand;
                break;
            }
        }
    }
    std::lock_guard<std::mutex> lk(mu);
    memo[key] = pick;
    return pick;
}

}  // namespace ann
}  // namespace sqs
