// Interval certifier of packings on the GPU, verdict for verdict and digit
// for digit the reference certifier (cuda/certifier.cpp:738-912).
//
// Pipeline of one batch:
//   host    envelope checks (row count, square ids), literal slices in
//           square-id order, optional pandas round-trip of every literal
//           (certifier.cpp:914-929), packings bucketed by n;
//   kernel  cert_packing_kernel, one CTA per packing:
//             literal syntax + exact double-range and bound checks
//             (certifier.cpp:764-791), Fix<9> side measurement with Taylor
//             sin/cos (:793-854), float corners + padded AABBs, bitonic sort
//             of the AABBs, sort-and-sweep with the float SAT prefilter
//             (:856-883); undecided pairs go to a global list;
//   kernel  cert_fp64_kernel: directed-rounding FP64 interval SAT of the
//           undecided pairs, deciding those whose sign it certifies (and
//           exact axis-aligned dyadic pairs) the way the stages below would;
//   kernels the 7-, 15- and 58-limb interval SAT of the pairs still open at
//           63, 135 and 522 decimal digits (:885-899), each stage taking the
//           pairs the previous one left open;
//   host    reason strings, area bound, score, 50-decimal side (:900-911).
// The kernel file is compiled without multiply-add contraction so its double
// arithmetic rounds exactly like the reference's host code.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "fixdev.cuh"

namespace sqs {
namespace cert {

using fx::Fix;
using fx::Iv;
using fx::Lit;

constexpr int kMaxN = 1000;
constexpr int kMaxLiteral = 100;
constexpr uint32_t kNoKey = 0xffffffffu;
constexpr unsigned long long kNoPair = ~0ull;

enum : uint32_t { kCertOverlap = 1u, kUndecidable = 2u, kPairOverflow = 4u };
enum : uint32_t { kErrParse = 0, kErrRange = 1, kErrCoord = 2, kErrAngle = 3 };

struct PkOut {
    uint32_t err_key;          // 4 * square + kind of the first failing check
    uint32_t flags;            // kCertOverlap | kUndecidable | kPairOverflow
    unsigned long long fkey;   // (ii << 32 | jj) of the first float overlap in sweep order
    int32_t fu, fv;            // that pair, as square ids
    uint32_t undecided;        // pairs sent to the interval stages
    uint32_t pad;
    Fix<9> side;               // max(span_x, span_y) of the corners, Fix<9>
};

struct Pair {
    int32_t pk;
    int16_t u, v;
};

struct Consts {
    Fix<9> half_pi9, two_pi9, half9;
    Fix<3> half3;
    Iv<7> half_pi7, half7;
    Iv<15> half_pi15, half15;
    Iv<58> half_pi58, half58;
};

__constant__ Consts c_consts;
// Decimal thresholds of the reference's double checks, exact:
//   strtod overflows      iff |v| >= 2^1024 - 2^970
//   |x| > 1e4 as a double iff |v| >  1e4 + 2^-40 (the tie rounds to 1e4)
//   |a| > 100 as a double iff |v| >  100 + 2^-47
__device__ const char c_inf_edge[] =
    "179769313486231580793728971405303415079934132710037826936173778980444968292764750946649017977587"
    "207096330286416692887910946555547851940402630657488671505820681908902000708383676273854845817711"
    "531764475730270069855571366959622842914819860834936475292719074168444365510704342711559699508093"
    "04222336";
__device__ const char c_coord_edge[] = "10000.0000000000009094947017729282379150390625";
__device__ const char c_angle_edge[] = "100.00000000000000710542735760100185871124267578125";

const char* kHalfPi =
    "1.5707963267948966192313216916397514420985846996875529104874722961539082031431044993140174126710585339"
    "9107404325664115332354692230477529111586267970406424055872514205135096926055277982231147447746519098"
    "2214405487832966723064237824116893391582635600954572824283161565386415559563044484210977355059400485"
    "7492389293099245510655716316154220989218499846888949675083019800051100514872368941154883214599416258"
    "7630228031340772652010253145121415210968393898212262598912242342639728019727481121132833606270987663"
    "3184560871636462872546121833290233099787539786414835847812261143213250625359595866490484368352035968";
const char* kTwoPi =
    "6.2831853071795864769252867665590057683943387987502116419498891846156328125724179972560696506842341359"
    "6429617302656461329418768921910116446345071881625696223490056820540387704221111928924589790986076392"
    "8857621951331866892256951296467573566330542403818291297132646261545662238252177936843909420237601942"
    "9969557172396982042622865264616883956873999387555798700332079200204402059489475764619532858397665035"
    "0520912125363090608041012580485660843873575592848905039564896937055891207890992448453133442508395065"
    "2738243486545851490184487333160932399150159145659343391249044572853002501438383465961937473408143872";

FX_HD bool is_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r'; }
FX_HD bool is_digit(char c) { return c >= '0' && c <= '9'; }

// is_valid_decimal (certifier.cpp:505-529) + the digit/point analysis of
// parse_decimal_fix (:265-333).  `base` is the text offset of `s`.
FX_HD bool analyze(const char* s, int len, uint32_t base, Lit& L, int max_len = kMaxLiteral) {
    int a = 0, b = len;
    while (a < b && is_space(s[a])) ++a;
    while (b > a && is_space(s[b - 1])) --b;
    const int n = b - a;
    L.off = base + (uint32_t)a;
    L.point = 0;
    L.ndig = 0;
    L.dot = -1;
    L.neg = 0;
    L.dyadic = 0;
    L.zero_str = 0;
    L.pad = 0;
    if (n <= 0 || n > max_len) return false;
    const char* t = s + a;
    int i = 0;
    if (t[0] == '+' || t[0] == '-') {
        L.neg = t[0] == '-';
        ++i;
    }
    if (i >= n) return false;
    L.off = base + (uint32_t)(a + i);
    bool any = false;
    int nd = 0, frac = 0;
    while (i < n && is_digit(t[i])) { any = true; ++i; ++nd; }
    if (i < n && t[i] == '.') {
        L.dot = (int16_t)nd;
        ++i;
        while (i < n && is_digit(t[i])) { any = true; ++i; ++nd; ++frac; }
    }
    if (!any) return false;
    long long ex = 0;
    if (i < n && (t[i] == 'e' || t[i] == 'E')) {
        ++i;
        int es = 1;
        if (i < n && (t[i] == '+' || t[i] == '-')) es = t[i++] == '-' ? -1 : 1;
        bool ed = false;
        while (i < n && is_digit(t[i])) {
            ed = true;
            if (ex < 100000000LL) ex = ex * 10 + (t[i] - '0');
            ++i;
        }
        if (!ed) return false;
        ex *= es;
    }
    if (i != n) return false;
    L.ndig = (uint16_t)nd;
    L.point = (int32_t)((long long)nd - frac + ex);
    L.zero_str = (n == 1 && t[0] == '0') || (n == 3 && t[0] == '0' && t[1] == '.' && t[2] == '0');
    return true;
}

// is_dyadic_decimal_str (certifier.cpp:335-381).
FX_HD bool dyadic(const char* text, const Lit& L) {
    int nd = L.ndig;
    long long places = (long long)L.ndig - L.point;
    while (places > 0 && nd > 0 && fx::lit_digit(text, L, nd - 1) == 0) { --nd; --places; }
    if (places <= 0) return true;
    if (places > 25) return false;
    char dg[kMaxLiteral + 4];
    int m = 0;
    for (int k = 0; k < nd; ++k) dg[m++] = (char)fx::lit_digit(text, L, k);
    for (long long k = 0; k < places; ++k) {
        if (m == 0) return true;
        if (dg[m - 1] % 5) return false;
        int rem = 0, w = 0;
        for (int r = 0; r < m; ++r) {
            const int cur = rem * 10 + dg[r];
            if (w > 0 || cur / 5) dg[w++] = (char)(cur / 5);
            rem = cur % 5;
        }
        m = w;
    }
    return true;
}

// Compare |literal| with a positive decimal constant (no sign, no exponent).
FX_HD int cmp_abs_const(const char* text, const Lit& L, const char* c) {
    int cl = 0, cdot = -1;
    while (c[cl]) {
        if (c[cl] == '.') cdot = cl;
        ++cl;
    }
    const int cint = cdot < 0 ? cl : cdot;           // constant's integer digit count
    const int cnd = cdot < 0 ? cl : cl - 1;
    auto cdig = [&](long long k) -> int {           // k-th digit of the constant
        if (k < 0 || k >= cnd) return 0;
        return c[(cdot >= 0 && k >= cdot) ? k + 1 : k] - '0';
    };
    int lz = 0;
    while (lz < L.ndig && fx::lit_digit(text, L, lz) == 0) ++lz;
    if (lz == L.ndig) return -1;  // zero
    const long long le = (long long)L.point - lz;    // digits before the point from the first non-zero
    int cz = 0;
    while (cz < cnd && cdig(cz) == 0) ++cz;
    const long long ce = (long long)cint - cz;
    if (le != ce) return le < ce ? -1 : 1;
    const long long len = (long long)(L.ndig - lz) > (long long)(cnd - cz) ? (L.ndig - lz) : (cnd - cz);
    for (long long k = 0; k < len; ++k) {
        const int a = fx::lit_digit(text, L, lz + k), b = cdig(cz + k);
        if (a != b) return a < b ? -1 : 1;
    }
    return 0;
}

// Float SAT prefilter (certifier.cpp:543-588) on squares with centre (x, y)
// and cached cos/sin (c, s) of the reduced angle.
struct FSq {
    double x, y, c, s;
};

__device__ __forceinline__ void fcorners(const FSq& q, double* cx, double* cy) {
    const double ux = 0.5 * q.c - 0.5 * q.s, uy = 0.5 * q.s + 0.5 * q.c;
    const double vx = -0.5 * q.c - 0.5 * q.s, vy = -0.5 * q.s + 0.5 * q.c;
    cx[0] = q.x + ux; cy[0] = q.y + uy;
    cx[1] = q.x + vx; cy[1] = q.y + vy;
    cx[2] = q.x - ux; cy[2] = q.y - uy;
    cx[3] = q.x - vx; cy[3] = q.y - vy;
}

__device__ __noinline__ int float_sat(const FSq& p, const FSq& q) {
    double px[4], py[4], qx[4], qy[4];
    fcorners(p, px, py);
    fcorners(q, qx, qy);
    const double ax[4][2] = {{p.c, p.s}, {-p.s, p.c}, {q.c, q.s}, {-q.s, q.c}};
    double worst = 1e300;
    for (int a = 0; a < 4; ++a) {
        double lo1 = 1e300, hi1 = -1e300, lo2 = 1e300, hi2 = -1e300;
        for (int k = 0; k < 4; ++k) {
            const double u = ax[a][0] * px[k] + ax[a][1] * py[k];
            const double v = ax[a][0] * qx[k] + ax[a][1] * qy[k];
            if (u < lo1) lo1 = u;
            if (u > hi1) hi1 = u;
            if (v < lo2) lo2 = v;
            if (v > hi2) hi2 = v;
        }
        const double ov = fmin(hi1, hi2) - fmax(lo1, lo2);
        if (ov < -1e-8) return 1;
        if (ov < worst) worst = ov;
    }
    return worst > 1e-8 ? -1 : 0;
}

template <int F>
__device__ void fix_shfl_min_max(Fix<F>& v, bool& have, bool want_min) {
    for (int o = 16; o > 0; o >>= 1) {
        Fix<F> w;
        for (int i = 0; i <= F; ++i) w.d[i] = __shfl_xor_sync(0xffffffffu, v.d[i], o);
        w.neg = __shfl_xor_sync(0xffffffffu, v.neg, o);
        const bool wh = __shfl_xor_sync(0xffffffffu, (int)have, o) != 0;
        if (wh && (!have || (want_min ? fx::cmp(w, v) < 0 : fx::cmp(w, v) > 0))) v = w;
        have = have || wh;
    }
}

// One CTA per packing: checks, side measurement, sort and sweep.
template <int T, int NMAX>
__global__ void __launch_bounds__(T, 512 / T) cert_packing_kernel(
    int count, const int32_t* __restrict__ bucket, const int32_t* __restrict__ pk_n,
    const int64_t* __restrict__ pk_sq0, const char* __restrict__ text, const int64_t* __restrict__ raw_off,
    const int32_t* __restrict__ raw_len, Lit* __restrict__ lits, PkOut* __restrict__ out,
    Pair* __restrict__ pairs, uint32_t* __restrict__ pair_count, uint32_t pair_cap) {
    constexpr int W = T / 32;
    constexpr int NP = NMAX;  // power of two
    extern __shared__ __align__(16) unsigned char dyn[];
    FSq* sq = reinterpret_cast<FSq*>(dyn);                    // by square id
    double* bx0 = reinterpret_cast<double*>(sq + NMAX);       // padded AABBs by square id
    double* bx1 = bx0 + NMAX;
    double* by0 = bx1 + NMAX;
    double* by1 = by0 + NMAX;
    double* key = by1 + NMAX;
    int16_t* idx = reinterpret_cast<int16_t*>(key + NP);
    __shared__ Fix<9> ext[W][4];
    __shared__ int ext_have[W];
    __shared__ Fix<9> org[2];
    __shared__ uint32_t s_err;
    __shared__ unsigned long long s_fkey;
    __shared__ uint32_t s_undecided;

    const int b = blockIdx.x;
    if (b >= count) return;
    const int pk = bucket[b];
    const int n = pk_n[pk];
    const int64_t s0 = pk_sq0[pk];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        s_err = kNoKey;
        s_fkey = kNoPair;
        s_undecided = 0;
    }
    __syncthreads();

    // 1. literal syntax and the double-range checks, first failure by square id
    for (int i = tid; i < n; i += T) {
        uint32_t kind = kNoKey;
        Lit Ls[3];
        for (int k = 0; k < 3; ++k) {
            const int64_t r = 3 * (s0 + i) + k;
            const bool ok = analyze(text + raw_off[r], raw_len[r], (uint32_t)raw_off[r], Ls[k]);
            if (!ok && kind == kNoKey) kind = kErrParse;
        }
        if (kind == kNoKey) {
            for (int k = 0; k < 3; ++k) {
                if (cmp_abs_const(text, Ls[k], c_inf_edge) >= 0) kind = kErrRange;
                Ls[k].dyadic = dyadic(text, Ls[k]);
            }
        }
        if (kind == kNoKey && (cmp_abs_const(text, Ls[0], c_coord_edge) > 0 ||
                               cmp_abs_const(text, Ls[1], c_coord_edge) > 0))
            kind = kErrCoord;
        if (kind == kNoKey && cmp_abs_const(text, Ls[2], c_angle_edge) > 0) kind = kErrAngle;
        for (int k = 0; k < 3; ++k) lits[3 * (s0 + i) + k] = Ls[k];
        if (kind != kNoKey) atomicMin(&s_err, 4u * (uint32_t)i + kind);
    }
    __syncthreads();
    if (s_err != kNoKey) {
        if (tid == 0) {
            out[pk].err_key = s_err;
            out[pk].fkey = kNoPair;
            out[pk].flags = 0;
            out[pk].undecided = 0;
        }
        return;
    }
    if (tid == 0) {
        org[0] = fx::parse<9>(text, lits[3 * s0], 0);
        org[1] = fx::parse<9>(text, lits[3 * s0 + 1], 0);
    }
    __syncthreads();

    // 2. Fix<9> corners (side) and float geometry, per square (the additions
    // and comparisons inlined; products, parsing and sin/cos out of line)
    Fix<9> mnx, mxx, mny, mxy;
    fx::set_zero(mnx);
    fx::set_zero(mxx);
    fx::set_zero(mny);
    fx::set_zero(mxy);
    bool have = false;
    const Consts& C = c_consts;
    for (int i = tid; i < n; i += T) {
        const Lit lx = lits[3 * (s0 + i)], ly = lits[3 * (s0 + i) + 1], la = lits[3 * (s0 + i) + 2];
        const Fix<9> X = fx::sub<9, true>(fx::parse<9>(text, lx, 0), org[0]);
        const Fix<9> Y = fx::sub<9, true>(fx::parse<9>(text, ly, 0), org[1]);
        const Fix<9> A = fx::parse<9>(text, la, 0);
        const long long turns = (long long)floor(fx::approx(A) / 6.283185307179586476925);
        Fix<9> red = fx::sub<9, true>(A, fx::mul(fx::of_int<9>(turns), C.two_pi9, 0));
        if (red.neg && !fx::is_zero(red)) red = fx::add<9, true>(red, C.two_pi9);
        if (fx::cmp<9, true>(red, C.two_pi9) >= 0) red = fx::sub<9, true>(red, C.two_pi9);
        FSq q;
        q.x = fx::approx(X);
        q.y = fx::approx(Y);
        const double ang = fx::approx(red);
        q.c = cos(ang);
        q.s = sin(ang);
        sq[i] = q;
        double cx[4], cy[4];
        fcorners(q, cx, cy);
        double x0 = cx[0], x1 = cx[0], y0 = cy[0], y1 = cy[0];
        for (int k = 1; k < 4; ++k) {
            x0 = fmin(x0, cx[k]); x1 = fmax(x1, cx[k]);
            y0 = fmin(y0, cy[k]); y1 = fmax(y1, cy[k]);
        }
        bx0[i] = x0 - 1e-7; by0[i] = y0 - 1e-7; bx1[i] = x1 + 1e-7; by1[i] = y1 + 1e-7;

        Fix<9> sn, cs;
        if (la.zero_str || fx::is_zero(A)) {
            cs = fx::of_int<9>(1);
            fx::set_zero(sn);
        } else {
            fx::sincos_point(A, C.half_pi9, sn, cs);
        }
        const Fix<9> hc = fx::mul(C.half9, cs, 0), hs = fx::mul(C.half9, sn, 0);
        const Fix<9> ux = fx::sub<9, true>(hc, hs), uy = fx::add<9, true>(hs, hc);
        Fix<9> zero;
        fx::set_zero(zero);
        const Fix<9> vx = fx::sub<9, true>(zero, fx::add<9, true>(hc, hs)), vy = fx::sub<9, true>(hc, hs);
        const Fix<9> px[4] = {fx::add<9, true>(X, ux), fx::add<9, true>(X, vx), fx::sub<9, true>(X, ux), fx::sub<9, true>(X, vx)};
        const Fix<9> py[4] = {fx::add<9, true>(Y, uy), fx::add<9, true>(Y, vy), fx::sub<9, true>(Y, uy), fx::sub<9, true>(Y, vy)};
        for (int k = 0; k < 4; ++k) {
            if (!have) {
                mnx = mxx = px[k];
                mny = mxy = py[k];
                have = true;
                continue;
            }
            if (fx::cmp<9, true>(px[k], mnx) < 0) mnx = px[k];
            if (fx::cmp<9, true>(px[k], mxx) > 0) mxx = px[k];
            if (fx::cmp<9, true>(py[k], mny) < 0) mny = py[k];
            if (fx::cmp<9, true>(py[k], mxy) > 0) mxy = py[k];
        }
    }
    {
        bool h0 = have, h1 = have, h2 = have, h3 = have;
        fix_shfl_min_max(mnx, h0, true);
        fix_shfl_min_max(mxx, h1, false);
        fix_shfl_min_max(mny, h2, true);
        fix_shfl_min_max(mxy, h3, false);
        if (lane == 0) {
            ext[warp][0] = mnx;
            ext[warp][1] = mxx;
            ext[warp][2] = mny;
            ext[warp][3] = mxy;
            ext_have[warp] = h0;
        }
    }
    // 3. sort the AABBs by their padded min x, ties by square id
    for (int i = tid; i < NP; i += T) {
        key[i] = i < n ? bx0[i] : 1e300;
        idx[i] = (int16_t)i;
    }
    __syncthreads();
    if (tid == 0) {
        Fix<9> e[4];
        bool any = false;
        for (int w = 0; w < W; ++w) {
            if (!ext_have[w]) continue;
            if (!any) {
                for (int k = 0; k < 4; ++k) e[k] = ext[w][k];
                any = true;
                continue;
            }
            if (fx::cmp(ext[w][0], e[0]) < 0) e[0] = ext[w][0];
            if (fx::cmp(ext[w][1], e[1]) > 0) e[1] = ext[w][1];
            if (fx::cmp(ext[w][2], e[2]) < 0) e[2] = ext[w][2];
            if (fx::cmp(ext[w][3], e[3]) > 0) e[3] = ext[w][3];
        }
        const Fix<9> sx = fx::sub(e[1], e[0]), sy = fx::sub(e[3], e[2]);
        out[pk].side = fx::cmp(sx, sy) >= 0 ? sx : sy;
    }
    int np = 1;
    while (np < n) np <<= 1;
    for (int k = 2; k <= np; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = tid; i < np; i += T) {
                const int l = i ^ j;
                if (l > i) {
                    const bool up = (i & k) == 0;
                    const double ki = key[i], kl = key[l];
                    const int16_t ii = idx[i], il = idx[l];
                    const bool gt = ki > kl || (ki == kl && ii > il);
                    if (gt == up) {
                        key[i] = kl; key[l] = ki;
                        idx[i] = il; idx[l] = ii;
                    }
                }
            }
            __syncthreads();
        }
    }

    // 4. sort and sweep with the float prefilter
    for (int ii = tid; ii < n; ii += T) {
        const int i = idx[ii];
        const double ix1 = bx1[i], iy0 = by0[i], iy1 = by1[i], ix0 = bx0[i];
        for (int jj = ii + 1; jj < n; ++jj) {
            const int j = idx[jj];
            if (bx0[j] > ix1) break;
            if (ix1 < bx0[j] || bx1[j] < ix0 || iy1 < by0[j] || by1[j] < iy0) continue;
            const int u = min(i, j), v = max(i, j);
            const int r = float_sat(sq[u], sq[v]);
            if (r < 0) {
                atomicMin(&s_fkey, ((unsigned long long)ii << 32) | (unsigned long long)jj);
            } else if (r == 0) {
                atomicAdd(&s_undecided, 1u);
                const uint32_t slot = atomicAdd(pair_count, 1u);
                if (slot < pair_cap) pairs[slot] = Pair{pk, (int16_t)u, (int16_t)v};
                else atomicOr(&out[pk].flags, kPairOverflow);
            }
        }
    }
    __syncthreads();
    if (tid == 0) {
        out[pk].err_key = kNoKey;
        out[pk].fkey = s_fkey;
        out[pk].undecided = s_undecided;
        if (s_fkey != kNoPair) {
            const int a = idx[(int)(s_fkey >> 32)], c = idx[(int)(s_fkey & 0xffffffffu)];
            out[pk].fu = min(a, c);
            out[pk].fv = max(a, c);
        }
    }
}

// ------------------------------------------------------------ interval stages
template <int F>
struct IvSq {
    bool flat;
    Iv<F> c, s, x0, x1, y0, y1;
    Iv<F> px[4], py[4];
};

template <int F>
__device__ __forceinline__ const Iv<F>& half_pi_iv();
template <>
__device__ __forceinline__ const Iv<7>& half_pi_iv<7>() { return c_consts.half_pi7; }
template <>
__device__ __forceinline__ const Iv<15>& half_pi_iv<15>() { return c_consts.half_pi15; }
template <>
__device__ __forceinline__ const Iv<58>& half_pi_iv<58>() { return c_consts.half_pi58; }
template <int F>
__device__ __forceinline__ const Iv<F>& half_iv();
template <>
__device__ __forceinline__ const Iv<7>& half_iv<7>() { return c_consts.half7; }
template <>
__device__ __forceinline__ const Iv<15>& half_iv<15>() { return c_consts.half15; }
template <>
__device__ __forceinline__ const Iv<58>& half_iv<58>() { return c_consts.half58; }

// ensure_sq_iv (certifier.cpp:600-635)
template <int F>
__device__ __noinline__ void make_ivsq(const char* text, const Lit* L3, const Iv<F>& ox, const Iv<F>& oy, IvSq<F>& e) {
    const Iv<F>& h = half_iv<F>();
    const Iv<F> x = fx::isub(fx::parse_iv<F>(text, L3[0]), ox);
    const Iv<F> y = fx::isub(fx::parse_iv<F>(text, L3[1]), oy);
    fx::sincos_iv(fx::parse_iv<F>(text, L3[2]), half_pi_iv<F>(), e.s, e.c);
    e.flat = fx::is_zero(e.s.lo) && fx::is_zero(e.s.hi);
    if (e.flat) {
        e.x0 = fx::isub(x, h);
        e.x1 = fx::iadd(x, h);
        e.y0 = fx::isub(y, h);
        e.y1 = fx::iadd(y, h);
    }
    const Iv<F> hc = fx::imul(h, e.c), hs = fx::imul(h, e.s), nh = fx::ineg(h);
    const Iv<F> ux = fx::isub(hc, hs), uy = fx::iadd(hs, hc);
    const Iv<F> vx = fx::isub(fx::imul(nh, e.c), hs), vy = fx::iadd(fx::imul(nh, e.s), hc);
    e.px[0] = fx::iadd(x, ux); e.py[0] = fx::iadd(y, uy);
    e.px[1] = fx::iadd(x, vx); e.py[1] = fx::iadd(y, vy);
    e.px[2] = fx::isub(x, ux); e.py[2] = fx::isub(y, uy);
    e.px[3] = fx::isub(x, vx); e.py[3] = fx::isub(y, vy);
}

// The interval SAT test runs for nearly every undecided pair: its comparisons,
// additions and subtractions are inlined at 7 limbs (fx::kInlineLimbs), the
// products stay out of line.
template <int F>
__device__ __forceinline__ Fix<F> fmin_(const Fix<F>& a, const Fix<F>& b) { return fx::cmp<F, true>(a, b) < 0 ? a : b; }
template <int F>
__device__ __forceinline__ Fix<F> fmax_(const Fix<F>& a, const Fix<F>& b) { return fx::cmp<F, true>(a, b) > 0 ? a : b; }

// sat_check_interval_cached (certifier.cpp:638-703)
template <int F>
__device__ __noinline__ int iv_sat(const IvSq<F>& p, const IvSq<F>& q) {
    Fix<F> z;
    fx::set_zero(z);
    if (p.flat && q.flat) {
        const Iv<F> ox = fx::isub<F, true>(Iv<F>{fmin_(p.x1.lo, q.x1.lo), fmin_(p.x1.hi, q.x1.hi)},
                                  Iv<F>{fmax_(p.x0.lo, q.x0.lo), fmax_(p.x0.hi, q.x0.hi)});
        if (fx::cmp<F, true>(ox.hi, z) <= 0) return 1;
        const Iv<F> oy = fx::isub<F, true>(Iv<F>{fmin_(p.y1.lo, q.y1.lo), fmin_(p.y1.hi, q.y1.hi)},
                                  Iv<F>{fmax_(p.y0.lo, q.y0.lo), fmax_(p.y0.hi, q.y0.hi)});
        if (fx::cmp<F, true>(oy.hi, z) <= 0) return 1;
        if (fx::cmp<F, true>(ox.lo, z) <= 0 || fx::cmp<F, true>(oy.lo, z) <= 0) return 0;
        return -1;
    }
    bool open = false;
    for (int a = 0; a < 4; ++a) {
        const IvSq<F>& o = a < 2 ? p : q;
        const Iv<F> ax = (a & 1) ? fx::ineg(o.s) : o.c;
        const Iv<F>& ay = (a & 1) ? o.c : o.s;
        Iv<F> mn1, mx1, mn2, mx2;
        for (int k = 0; k < 4; ++k) {
            const Iv<F> u = fx::iadd<F, true>(fx::imul(ax, p.px[k]), fx::imul(ay, p.py[k]));
            const Iv<F> v = fx::iadd<F, true>(fx::imul(ax, q.px[k]), fx::imul(ay, q.py[k]));
            if (k == 0) {
                mn1 = mx1 = u;
                mn2 = mx2 = v;
                continue;
            }
            mn1.lo = fmin_(u.lo, mn1.lo); mn1.hi = fmin_(u.hi, mn1.hi);
            mx1.lo = fmax_(u.lo, mx1.lo); mx1.hi = fmax_(u.hi, mx1.hi);
            mn2.lo = fmin_(v.lo, mn2.lo); mn2.hi = fmin_(v.hi, mn2.hi);
            mx2.lo = fmax_(v.lo, mx2.lo); mx2.hi = fmax_(v.hi, mx2.hi);
        }
        const Iv<F> ov = fx::isub<F, true>(Iv<F>{fmin_(mx1.lo, mx2.lo), fmin_(mx1.hi, mx2.hi)},
                                  Iv<F>{fmax_(mn1.lo, mn2.lo), fmax_(mn1.hi, mn2.hi)});
        if (fx::cmp<F, true>(ov.hi, z) <= 0) return 1;
        if (fx::cmp<F, true>(ov.lo, z) <= 0) open = true;
    }
    return open ? 0 : -1;
}

template <int F>
__global__ void __launch_bounds__(128) cert_stage_kernel(
    const Pair* __restrict__ in, const uint32_t* __restrict__ in_count, uint32_t in_cap,
    Pair* __restrict__ next, uint32_t* __restrict__ next_count, uint32_t next_cap,
    const int64_t* __restrict__ pk_sq0, const Lit* __restrict__ lits, const char* __restrict__ text,
    PkOut* __restrict__ out) {
    const uint32_t total = min(*in_count, in_cap);
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const Pair pr = in[t];
        PkOut& po = out[pr.pk];
        if (po.fkey != kNoPair || (po.flags & kCertOverlap)) continue;
        const int64_t s0 = pk_sq0[pr.pk];
        const Iv<F> ox = fx::parse_iv<F>(text, lits[3 * s0]);
        const Iv<F> oy = fx::parse_iv<F>(text, lits[3 * s0 + 1]);
        IvSq<F> A, Bq;
        make_ivsq<F>(text, lits + 3 * (s0 + pr.u), ox, oy, A);
        make_ivsq<F>(text, lits + 3 * (s0 + pr.v), ox, oy, Bq);
        const int r = iv_sat<F>(A, Bq);
        if (r < 0) {
            atomicOr(&po.flags, kCertOverlap);
        } else if (r == 0) {
            if (next == nullptr) {
                atomicOr(&po.flags, kUndecidable);
            } else {
                const uint32_t slot = atomicAdd(next_count, 1u);
                if (slot < next_cap) next[slot] = pr;
                else atomicOr(&po.flags, kPairOverflow);
            }
        }
    }
}

// ------------------------------------------------------------ FP64 prefilter
// Directed-rounding FP64 interval SAT of the pairs the float check left open,
// ahead of the multi-limb stages.  It decides a pair only where those stages
// are certain to decide it the same way, so verdicts stay the reference's:
//   * separated (1) when some axis's overlap interval lies strictly below
//     zero, overlapping (-1) when every axis's lies strictly above: the
//     intervals enclose the exact overlap of the exact decimal inputs, so its
//     sign is certain, and an exact value of |v| >= 2^-1074 is resolved the
//     same way by the 7-, 15- or 58-limb stage (widths below 1e-60);
//   * two axis-aligned squares (angle literal exactly zero, the reference's
//     flat path) whose coordinate literals and square 0's are all dyadic
//     within 25 decimal places are compared exactly in 3-limb fixed point,
//     the values the 7-limb stage computes exactly: touching edges decide
//     as separated, as they do there;
//   * everything else goes on to the 7-limb stage.
// Bounds: a literal's value from its 27-decimal truncation (error < 1e-27)
// converted to double (error below (|v| + 1) 2^-47), widened by both; sin
// and cos from CUDA's double sincos, whose documented error is 2 ulp
// (below 2^-51 in [-1, 1]), widened by that and by the angle's half-width.
struct DIv {
    double lo, hi;
};
__device__ __forceinline__ DIv d_add(DIv a, DIv b) { return DIv{__dadd_rd(a.lo, b.lo), __dadd_ru(a.hi, b.hi)}; }
__device__ __forceinline__ DIv d_sub(DIv a, DIv b) { return DIv{__dsub_rd(a.lo, b.hi), __dsub_ru(a.hi, b.lo)}; }
__device__ __forceinline__ DIv d_mul(DIv a, DIv b) {
    const double l0 = __dmul_rd(a.lo, b.lo), l1 = __dmul_rd(a.lo, b.hi), l2 = __dmul_rd(a.hi, b.lo),
                 l3 = __dmul_rd(a.hi, b.hi);
    const double h0 = __dmul_ru(a.lo, b.lo), h1 = __dmul_ru(a.lo, b.hi), h2 = __dmul_ru(a.hi, b.lo),
                 h3 = __dmul_ru(a.hi, b.hi);
    return DIv{fmin(fmin(l0, l1), fmin(l2, l3)), fmax(fmax(h0, h1), fmax(h2, h3))};
}
__device__ __forceinline__ DIv d_half(DIv a) { return DIv{0.5 * a.lo, 0.5 * a.hi}; }  // exact
__device__ __forceinline__ DIv d_neg(DIv a) { return DIv{-a.hi, -a.lo}; }

// Enclosure of a literal's exact value.
__device__ __forceinline__ DIv lit_iv(const char* text, const Lit& L) {
    const double a = fx::approx(fx::parse<3>(text, L, 0));
    const double eps = __dadd_ru(__dmul_ru(__dadd_ru(fabs(a), 1.0), 0x1p-47), 1e-27);
    return DIv{__dsub_rd(a, eps), __dadd_ru(a, eps)};
}

__device__ __forceinline__ bool lit_is_zero(const char* text, const Lit& L) {
    for (int k = 0; k < L.ndig; ++k)
        if (fx::lit_digit(text, L, k) != 0) return false;
    return true;
}

struct DSq {
    bool flat;
    DIv c, s, X, Y;
    DIv px[4], py[4];
};

__device__ __noinline__ void make_dsq(const char* text, const Lit* L3, DIv ox, DIv oy, DSq& e) {
    e.X = d_sub(lit_iv(text, L3[0]), ox);
    e.Y = d_sub(lit_iv(text, L3[1]), oy);
    e.flat = lit_is_zero(text, L3[2]);
    if (e.flat) {
        e.c = DIv{1.0, 1.0};
        e.s = DIv{0.0, 0.0};
    } else {
        const DIv a = lit_iv(text, L3[2]);
        const double mid = 0.5 * (a.lo + a.hi);
        double sn, cs;
        sincos(mid, &sn, &cs);
        const double w = __dadd_ru(0x1p-50, __dsub_ru(a.hi, a.lo));
        e.c = DIv{__dsub_rd(cs, w), __dadd_ru(cs, w)};
        e.s = DIv{__dsub_rd(sn, w), __dadd_ru(sn, w)};
    }
    const DIv hc = d_half(e.c), hs = d_half(e.s);
    const DIv ux = d_sub(hc, hs), uy = d_add(hs, hc);
    const DIv vx = d_sub(d_neg(hc), hs), vy = d_add(d_neg(hs), hc);
    e.px[0] = d_add(e.X, ux); e.py[0] = d_add(e.Y, uy);
    e.px[1] = d_add(e.X, vx); e.py[1] = d_add(e.Y, vy);
    e.px[2] = d_sub(e.X, ux); e.py[2] = d_sub(e.Y, uy);
    e.px[3] = d_sub(e.X, vx); e.py[3] = d_sub(e.Y, vy);
}

// Exact box test of two axis-aligned squares with dyadic literals (the
// reference's flat path on exact values): 1 separated or touching, -1 overlapping.
__device__ __noinline__ int exact_flat_sat(const char* text, const Lit* P, const Lit* Q, const Lit* O) {
    using F3 = Fix<3>;
    const F3 ox = fx::parse<3>(text, O[0], 0), oy = fx::parse<3>(text, O[1], 0);
    const F3 h = c_consts.half3;
    const F3 px = fx::sub(fx::parse<3>(text, P[0], 0), ox), py = fx::sub(fx::parse<3>(text, P[1], 0), oy);
    const F3 qx = fx::sub(fx::parse<3>(text, Q[0], 0), ox), qy = fx::sub(fx::parse<3>(text, Q[1], 0), oy);
    auto mn = [](const F3& a, const F3& b) { return fx::cmp(a, b) < 0 ? a : b; };
    auto mx = [](const F3& a, const F3& b) { return fx::cmp(a, b) > 0 ? a : b; };
    F3 z;
    fx::set_zero(z);
    const F3 ovx = fx::sub(mn(fx::add(px, h), fx::add(qx, h)), mx(fx::sub(px, h), fx::sub(qx, h)));
    if (fx::cmp(ovx, z) <= 0) return 1;
    const F3 ovy = fx::sub(mn(fx::add(py, h), fx::add(qy, h)), mx(fx::sub(py, h), fx::sub(qy, h)));
    if (fx::cmp(ovy, z) <= 0) return 1;
    return -1;
}

// 1 separated, -1 overlapping, 0 left to the multi-limb stages.
__device__ __noinline__ int fp64_sat(const DSq& p, const DSq& q) {
    if (p.flat && q.flat) {
        const DIv ox = DIv{__dsub_rd(fmin(__dadd_rd(p.X.lo, 0.5), __dadd_rd(q.X.lo, 0.5)),
                                     fmax(__dsub_ru(p.X.hi, 0.5), __dsub_ru(q.X.hi, 0.5))),
                           __dsub_ru(fmin(__dadd_ru(p.X.hi, 0.5), __dadd_ru(q.X.hi, 0.5)),
                                     fmax(__dsub_rd(p.X.lo, 0.5), __dsub_rd(q.X.lo, 0.5)))};
        const DIv oy = DIv{__dsub_rd(fmin(__dadd_rd(p.Y.lo, 0.5), __dadd_rd(q.Y.lo, 0.5)),
                                     fmax(__dsub_ru(p.Y.hi, 0.5), __dsub_ru(q.Y.hi, 0.5))),
                           __dsub_ru(fmin(__dadd_ru(p.Y.hi, 0.5), __dadd_ru(q.Y.hi, 0.5)),
                                     fmax(__dsub_rd(p.Y.lo, 0.5), __dsub_rd(q.Y.lo, 0.5)))};
        if (ox.hi < 0.0 || oy.hi < 0.0) return 1;
        if (ox.lo > 0.0 && oy.lo > 0.0) return -1;
        return 0;
    }
    bool all_pos = true;
    for (int a = 0; a < 4; ++a) {
        const DSq& o = a < 2 ? p : q;
        const DIv ax = (a & 1) ? d_neg(o.s) : o.c, ay = (a & 1) ? o.c : o.s;
        DIv mn1{1e300, 1e300}, mx1{-1e300, -1e300}, mn2{1e300, 1e300}, mx2{-1e300, -1e300};
        for (int k = 0; k < 4; ++k) {
            const DIv u = d_add(d_mul(ax, p.px[k]), d_mul(ay, p.py[k]));
            const DIv v = d_add(d_mul(ax, q.px[k]), d_mul(ay, q.py[k]));
            mn1 = DIv{fmin(mn1.lo, u.lo), fmin(mn1.hi, u.hi)};
            mx1 = DIv{fmax(mx1.lo, u.lo), fmax(mx1.hi, u.hi)};
            mn2 = DIv{fmin(mn2.lo, v.lo), fmin(mn2.hi, v.hi)};
            mx2 = DIv{fmax(mx2.lo, v.lo), fmax(mx2.hi, v.hi)};
        }
        const DIv ov = d_sub(DIv{fmin(mx1.lo, mx2.lo), fmin(mx1.hi, mx2.hi)},
                             DIv{fmax(mn1.lo, mn2.lo), fmax(mn1.hi, mn2.hi)});
        if (ov.hi < 0.0) return 1;
        all_pos &= ov.lo > 0.0;
    }
    return all_pos ? -1 : 0;
}

__global__ void __launch_bounds__(128) cert_fp64_kernel(const Pair* __restrict__ in, const uint32_t* __restrict__ in_count,
                                                        uint32_t in_cap, Pair* __restrict__ next,
                                                        uint32_t* __restrict__ next_count, uint32_t next_cap,
                                                        const int64_t* __restrict__ pk_sq0,
                                                        const Lit* __restrict__ lits, const char* __restrict__ text,
                                                        PkOut* __restrict__ out) {
    const uint32_t total = min(*in_count, in_cap);
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const Pair pr = in[t];
        PkOut& po = out[pr.pk];
        if (po.fkey != kNoPair || (po.flags & kCertOverlap)) continue;
        const int64_t s0 = pk_sq0[pr.pk];
        const Lit* O = lits + 3 * s0;
        const Lit* P = lits + 3 * (s0 + pr.u);
        const Lit* Q = lits + 3 * (s0 + pr.v);
        int r;
        if (lit_is_zero(text, P[2]) && lit_is_zero(text, Q[2]) && O[0].dyadic && O[1].dyadic && P[0].dyadic &&
            P[1].dyadic && Q[0].dyadic && Q[1].dyadic) {
            r = exact_flat_sat(text, P, Q, O);
        } else {
            const DIv ox = lit_iv(text, O[0]), oy = lit_iv(text, O[1]);
            DSq A, B;
            make_dsq(text, P, ox, oy, A);
            make_dsq(text, Q, ox, oy, B);
            r = fp64_sat(A, B);
        }
        if (r < 0) {
            atomicOr(&po.flags, kCertOverlap);
        } else if (r == 0) {
            const uint32_t slot = atomicAdd(next_count, 1u);
            if (slot < next_cap) next[slot] = pr;
            else atomicOr(&po.flags, kPairOverflow);
        }
    }
}

// ------------------------------------------------------------ cached stages
// The same interval test with every square's interval corners computed once
// per stage, as the reference caches them per square (ensure_sq_iv,
// certifier.cpp:600-635): a square sits in about four undecided pairs of a
// contact-heavy packing, and its parse + Taylor sin/cos is the expensive part.
//   mark   claims a cache slot for each square of a live pair (one claim per
//          square: slot_of[] holds -1, then -2 while claimed, then the slot);
//   build  one thread per claimed square writes its IvSq<F> to the cache in
//          HBM;
//   pair   one thread per pair runs iv_sat on references into the cache.
// Flags only ever get set, so a pair the mark kernel skipped (its packing
// already decided) is skipped by the pair kernel too.
struct SqRef {
    int32_t sq;  // global square index (packing's first square + id)
    int32_t pk;
};

__device__ __forceinline__ bool pair_live(const PkOut& po) {
    return po.fkey == kNoPair && !(po.flags & kCertOverlap);
}

__global__ void __launch_bounds__(256) cert_mark_kernel(const Pair* __restrict__ in, const uint32_t* __restrict__ in_count,
                                                       uint32_t in_cap, const int64_t* __restrict__ pk_sq0,
                                                       int32_t* __restrict__ slot_of, SqRef* __restrict__ list,
                                                       uint32_t* __restrict__ list_count, uint32_t list_cap,
                                                       PkOut* __restrict__ out) {
    const uint32_t total = min(*in_count, in_cap);
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const Pair pr = in[t];
        if (!pair_live(out[pr.pk])) continue;
        const int64_t s0 = pk_sq0[pr.pk];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int32_t g = (int32_t)(s0 + (k ? pr.v : pr.u));
            if (atomicCAS(&slot_of[g], -1, -2) == -1) {
                const uint32_t slot = atomicAdd(list_count, 1u);
                if (slot < list_cap) {
                    list[slot] = SqRef{g, pr.pk};
                    slot_of[g] = (int32_t)slot;
                } else {
                    atomicOr(&out[pr.pk].flags, kPairOverflow);
                }
            }
        }
    }
}

template <int F>
__global__ void __launch_bounds__(128) cert_build_kernel(const SqRef* __restrict__ list,
                                                        const uint32_t* __restrict__ list_count, uint32_t list_cap,
                                                        const int64_t* __restrict__ pk_sq0,
                                                        const Lit* __restrict__ lits, const char* __restrict__ text,
                                                        IvSq<F>* __restrict__ cache) {
    const uint32_t total = min(*list_count, list_cap);
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const SqRef r = list[t];
        const int64_t s0 = pk_sq0[r.pk];
        const Iv<F> ox = fx::parse_iv<F>(text, lits[3 * s0]);
        const Iv<F> oy = fx::parse_iv<F>(text, lits[3 * s0 + 1]);
        make_ivsq<F>(text, lits + 3 * (int64_t)r.sq, ox, oy, cache[t]);
    }
}

template <int F>
__global__ void __launch_bounds__(128) cert_pair_kernel(const Pair* __restrict__ in,
                                                       const uint32_t* __restrict__ in_count, uint32_t in_cap,
                                                       Pair* __restrict__ next, uint32_t* __restrict__ next_count,
                                                       uint32_t next_cap, const int64_t* __restrict__ pk_sq0,
                                                       const int32_t* __restrict__ slot_of,
                                                       const IvSq<F>* __restrict__ cache, PkOut* __restrict__ out) {
    const uint32_t total = min(*in_count, in_cap);
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const Pair pr = in[t];
        PkOut& po = out[pr.pk];
        if (!pair_live(po)) continue;
        const int64_t s0 = pk_sq0[pr.pk];
        const int32_t a = slot_of[s0 + pr.u], b = slot_of[s0 + pr.v];
        if (a < 0 || b < 0) {  // no cache entry (the slot list overflowed): report, never guess
            atomicOr(&po.flags, kPairOverflow);
            continue;
        }
        const int r = iv_sat<F>(cache[a], cache[b]);
        if (r < 0) {
            atomicOr(&po.flags, kCertOverlap);
        } else if (r == 0) {
            if (next == nullptr) {
                atomicOr(&po.flags, kUndecidable);
            } else {
                const uint32_t slot = atomicAdd(next_count, 1u);
                if (slot < next_cap) next[slot] = pr;
                else atomicOr(&po.flags, kPairOverflow);
            }
        }
    }
}

// ------------------------------------------------------------ host side
// Constants (600-digit pi/2, 2 pi) are analysed without the 100-character
// literal limit that applies to submitted coordinates.
static int host_lit(const char* s, Lit& L) {
    if (!analyze(s, (int)std::strlen(s), 0, L, 1 << 20)) {
        set_error("internal: constant literal does not parse");
        return SQS_EINVAL;
    }
    L.dyadic = dyadic(s, L);
    return SQS_OK;
}

// Literal texts of this size range are staged in pinned memory for the
// upload (larger ones are uploaded from the caller's memory, rather than
// pinning gigabytes of host memory).
constexpr size_t kPinnedTextMin = (size_t)4 << 20;
constexpr size_t kPinnedTextMax = (size_t)1 << 30;

static int upload_consts(int device) {
    static std::atomic<bool> done[64];
    static std::mutex mu;  // several host threads may certify at once
    if (done[device & 63]) return SQS_OK;
    std::lock_guard<std::mutex> lk(mu);
    if (done[device & 63]) return SQS_OK;
    Consts c;
    Lit hp, tp, h;
    if (int r = host_lit(kHalfPi, hp)) return r;
    if (int r = host_lit(kTwoPi, tp)) return r;
    if (int r = host_lit("0.5", h)) return r;
    c.half_pi9 = fx::parse<9>(kHalfPi, hp, 0);
    c.two_pi9 = fx::parse<9>(kTwoPi, tp, 0);
    c.half9 = fx::parse<9>("0.5", h, 0);
    c.half3 = fx::parse<3>("0.5", h, 0);
    c.half_pi7 = fx::parse_iv<7>(kHalfPi, hp);
    c.half7 = fx::parse_iv<7>("0.5", h);
    c.half_pi15 = fx::parse_iv<15>(kHalfPi, hp);
    c.half15 = fx::parse_iv<15>("0.5", h);
    c.half_pi58 = fx::parse_iv<58>(kHalfPi, hp);
    c.half58 = fx::parse_iv<58>("0.5", h);
    SQS_CUDA(cudaMemcpyToSymbol(c_consts, &c, sizeof c));
    done[device & 63] = true;
    return SQS_OK;
}

// The side rounded half-to-even at 50 decimals (format_50_decimals,
// certifier.cpp:60-104), written into dst (cap >= 80 holds every side here).
static void fifty_into(const Fix<9>& v, char* dst, size_t cap) {
    const uint64_t B = 1000000000ULL;
    uint64_t low = v.d[6] % 10000ULL, top = v.d[6] / 10000ULL;
    const bool tail = v.d[7] || v.d[8] || v.d[9];
    const bool up = low > 5000ULL || (low == 5000ULL && (tail || (top & 1ULL)));
    uint64_t o[7] = {v.d[0], v.d[1], v.d[2], v.d[3], v.d[4], v.d[5], top};
    if (up && ++o[6] >= 100000ULL) {
        o[6] -= 100000ULL;
        int i = 5;
        for (; i >= 1; --i) {
            if (++o[i] < B) break;
            o[i] -= B;
        }
        if (i < 1) o[0] += 1;
    }
    bool allz = true;
    for (uint64_t w : o) allz &= w == 0;
    std::snprintf(dst, cap, "%s%llu.%09llu%09llu%09llu%09llu%09llu%05llu", (v.neg && !allz) ? "-" : "",
                  (unsigned long long)o[0], (unsigned long long)o[1], (unsigned long long)o[2],
                  (unsigned long long)o[3], (unsigned long long)o[4], (unsigned long long)o[5],
                  (unsigned long long)o[6]);
}

static std::string fifty(const Fix<9>& v) {
    char buf[128];
    fifty_into(v, buf, sizeof buf);
    return buf;
}

static double grid_score(int n) { return std::ceil(std::sqrt((double)n)) / std::sqrt((double)n) - 1.0; }

// The pandas float round trip of one value (roundtrip_float_str,
// certifier.cpp:914-929): the shortest of %.15g, %.16g, %.17g that reads back
// as v, with ".0" appended to a plain integer; returns its length (< 40).
static size_t roundtrip_into(double v, char out[40]) {
    for (int p = 15; p <= 17; ++p) {
        std::snprintf(out, 40, "%.*g", p, v);
        if (std::strtod(out, nullptr) == v) break;
    }
    size_t len = std::strlen(out);
    if (std::strpbrk(out, ".eE") == nullptr) {
        std::memcpy(out + len, ".0", 3);
        len += 2;
    }
    return len;
}

static std::string roundtrip(const char* s, size_t len) {
    std::string in(s, len);
    char buf[40];
    const size_t k = roundtrip_into(std::strtod(in.c_str(), nullptr), buf);
    return std::string(buf, k);
}

static void put(char* dst, size_t cap, const std::string& s) {
    size_t k = std::min(cap - 1, s.size());
    std::memcpy(dst, s.data(), k);
    dst[k] = 0;
}

template <int T, int NMAX>
static int launch_packing(sqs_ctx* ctx, int count, const int32_t* bucket, const int32_t* pk_n,
                          const int64_t* pk_sq0, const char* text, const int64_t* raw_off,
                          const int32_t* raw_len, Lit* lits, PkOut* out, Pair* pairs, uint32_t* pair_count,
                          uint32_t cap) {
    if (count == 0) return SQS_OK;
    const size_t smem = (size_t)NMAX * (sizeof(FSq) + 5 * sizeof(double) + sizeof(int16_t));
    static std::atomic<bool> attr[64];  // set-up once per device (idempotent if repeated)
    if (!attr[ctx->device & 63]) {
        SQS_CUDA(cudaFuncSetAttribute(cert_packing_kernel<T, NMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
        attr[ctx->device & 63] = true;
    }
    cert_packing_kernel<T, NMAX><<<count, T, smem, ctx->stream>>>(count, bucket, pk_n, pk_sq0, text, raw_off,
                                                               raw_len, lits, out, pairs, pair_count, cap);
    SQS_CUDA(cudaGetLastError());
    ctx->launches += 1;
    return SQS_OK;
}

template <int F>
static int launch_stage(sqs_ctx* ctx, const Pair* in, const uint32_t* in_count, uint32_t in_cap, Pair* next,
                        uint32_t* next_count, uint32_t next_cap, const int64_t* pk_sq0, const Lit* lits,
                        const char* text, PkOut* out, int blocks) {
    cert_stage_kernel<F><<<blocks, 128, 0, ctx->stream>>>(in, in_count, in_cap, next, next_count, next_cap,
                                                         pk_sq0, lits, text, out);
    SQS_CUDA(cudaGetLastError());
    ctx->launches += 1;
    return SQS_OK;
}

// The FP64 prefilter over a pair list (grid-stride; the count stays on the device).
static int launch_fp64(sqs_ctx* ctx, const Pair* in, const uint32_t* in_count, uint32_t in_cap, Pair* next,
                       uint32_t* next_count, uint32_t next_cap, const int64_t* pk_sq0, const Lit* lits,
                       const char* text, PkOut* out, int blocks) {
    cert_fp64_kernel<<<blocks, 128, 0, ctx->stream>>>(in, in_count, in_cap, next, next_count, next_cap, pk_sq0, lits,
                                                       text, out);
    SQS_CUDA(cudaGetLastError());
    ctx->launches += 1;
    return SQS_OK;
}

static unsigned grid_for(sqs_ctx* ctx, uint32_t items, unsigned threads) {
    const uint64_t want = ((uint64_t)items + threads - 1) / threads;
    const uint64_t cap = (uint64_t)ctx->sm_count * 8;
    return (unsigned)std::max<uint64_t>(1, std::min(want, cap));
}

// One escalation stage with the per-square cache.  Reads back the stage's
// pair count (a stage without pairs launches nothing) and the number of
// claimed squares (the cache is sized to exactly those).
template <int F>
static int cached_stage(sqs_ctx* ctx, const Pair* in, const uint32_t* in_count, uint32_t cap, Pair* next,
                        uint32_t* next_count, const int64_t* d_s0, const Lit* d_lits, const char* d_text,
                        PkOut* d_out, int32_t* slot_of, SqRef* list, uint32_t* list_count, int64_t S) {
    uint32_t h_in = 0;
    SQS_CUDA(cudaMemcpyAsync(&h_in, in_count, 4, cudaMemcpyDeviceToHost, ctx->stream));
    SQS_CUDA(cudaStreamSynchronize(ctx->stream));
    h_in = std::min(h_in, cap);
    if (h_in == 0) return SQS_OK;
    const uint32_t list_cap = (uint32_t)std::min<int64_t>(S, 2ll * h_in);
    SQS_CUDA(cudaMemsetAsync(slot_of, 0xff, (size_t)S * sizeof(int32_t), ctx->stream));
    SQS_CUDA(cudaMemsetAsync(list_count, 0, sizeof(uint32_t), ctx->stream));
    cert_mark_kernel<<<grid_for(ctx, h_in, 256), 256, 0, ctx->stream>>>(in, in_count, cap, d_s0, slot_of, list,
                                                                         list_count, list_cap, d_out);
    SQS_CUDA(cudaGetLastError());
    ctx->launches += 1;
    uint32_t h_sq = 0;
    SQS_CUDA(cudaMemcpyAsync(&h_sq, list_count, 4, cudaMemcpyDeviceToHost, ctx->stream));
    SQS_CUDA(cudaStreamSynchronize(ctx->stream));
    h_sq = std::min(h_sq, list_cap);
    IvSq<F>* cache = nullptr;
    if (h_sq > 0) {
        if (int r = ctx->d_cert.reserve((size_t)h_sq * sizeof(IvSq<F>))) return r;
        cache = (IvSq<F>*)ctx->d_cert.p;
        cert_build_kernel<F><<<grid_for(ctx, h_sq, 128), 128, 0, ctx->stream>>>(list, list_count, list_cap, d_s0,
                                                                                 d_lits, d_text, cache);
        SQS_CUDA(cudaGetLastError());
        ctx->launches += 1;
    }
    cert_pair_kernel<F><<<grid_for(ctx, h_in, 128), 128, 0, ctx->stream>>>(
        in, in_count, cap, next, next_count, next ? cap : 0, d_s0, slot_of, cache, d_out);
    SQS_CUDA(cudaGetLastError());
    ctx->launches += 1;
    return SQS_OK;
}

}  // namespace cert
}  // namespace sqs

using namespace sqs;
using namespace sqs::cert;

extern "C" int sqs_certify_batch(sqs_ctx* ctx, int count, const int32_t* n_of, const int64_t* row_start,
                                 const int32_t* square_id, const char* text, const int64_t* lit_off, int flags,
                                 sqs_verdict* out) {
    if (int r = enter(ctx)) return r;
    SQS_REQUIRE(count >= 0, "count %d < 0", count);
    if (count == 0) return SQS_OK;
    SQS_REQUIRE(n_of && row_start && text && lit_off && out, "null host pointer");
    if (int r = upload_consts(ctx->device)) return r;

    // 1. the envelope of every packing (serial, cheap): verdict defaults, row
    //    counts, and the square offsets of those that may certify
    std::vector<int32_t> pk_n((size_t)count, 0);
    std::vector<int64_t> pk_sq0((size_t)count, 0);
    std::vector<char> live((size_t)count, 0);
    const bool do_rt = (flags & SQS_CERT_ROUNDTRIP) != 0;
    int64_t S = 0;
    for (int p = 0; p < count; ++p) {
        const int n = n_of[p];
        sqs_verdict& v = out[p];
        std::memset(&v, 0, sizeof v);
        v.n = n;
        SQS_REQUIRE(n >= 1 && n <= kMaxN, "packing %d: n=%d out of 1..%d", p, n, kMaxN);
        v.score = grid_score(n);
        const int64_t r0 = row_start[p], r1 = row_start[p + 1];
        SQS_REQUIRE(r1 >= r0, "packing %d: row_start not monotone", p);
        if (r1 - r0 != n) {
            const std::string N = std::to_string(n);
            put(v.reason, sizeof v.reason, "n=" + N + ": expected " + N + " rows, got " + std::to_string(r1 - r0));
            continue;
        }
        live[(size_t)p] = 1;
        pk_n[(size_t)p] = n;
        pk_sq0[(size_t)p] = S;
        S += n;
    }
    SQS_REQUIRE(S < (1ll << 30), "%lld squares in one call (limit 2^30)", (long long)S);
    // 2. square ids and literal slices (round-tripped when asked), host
    //    threads over contiguous ranges of packings with equal square counts
    // Literal slice tables, written straight into the context's pinned
    // staging: no zero fill, no page faults after the first call, and an
    // upload at the full host-link rate.  Every slot of a live packing is
    // written below; slots of packings found invalid are never read.
    const size_t n3 = (size_t)(3 * S);
    if (int r = ctx->h_cert.reserve(n3 * (sizeof(int64_t) + sizeof(int32_t)) + 16)) return r;
    int64_t* const raw_off = (int64_t*)ctx->h_cert.p;
    int32_t* const raw_len = (int32_t*)(raw_off + n3);
    const int nt = count >= 64 ? (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency())) : 1;
    std::vector<int> p_lo((size_t)nt + 1, count);
    {
        int t = 0;
        p_lo[0] = 0;
        for (int p = 0; p < count && t + 1 < nt; ++p)
            if (pk_sq0[(size_t)p] >= (S * (t + 1)) / nt) p_lo[(size_t)++t] = p;
        for (++t; t <= nt; ++t) p_lo[(size_t)t] = count;
    }
    std::vector<std::string> rt((size_t)nt);  // round-tripped text of each thread's packings
    std::vector<int64_t> bad_row((size_t)nt, -1);
    // A large literal text is staged in pinned memory too, each thread copying
    // the span of its own packings (the first from offset 0), so that it
    // uploads at the full host-link rate.
    const size_t text_bytes = (size_t)lit_off[3 * row_start[count]];
    char* h_text = nullptr;
    if (!do_rt && text_bytes >= kPinnedTextMin && text_bytes <= kPinnedTextMax) {
        if (int r = ctx->h_text.reserve(text_bytes)) return r;
        h_text = (char*)ctx->h_text.p;
    }
    auto slice = [&](int t) {
        if (h_text) {
            const int64_t a = t == 0 ? 0 : lit_off[3 * row_start[p_lo[(size_t)t]]];
            const int64_t b = t + 1 == nt ? (int64_t)text_bytes : lit_off[3 * row_start[p_lo[(size_t)t + 1]]];
            if (b > a && a >= 0 && (size_t)b <= text_bytes) std::memcpy(h_text + a, text + a, (size_t)(b - a));
        }
        std::vector<int64_t> row_of;
        for (int p = p_lo[(size_t)t]; p < p_lo[(size_t)t + 1]; ++p) {
            if (!live[(size_t)p]) continue;
            const int n = pk_n[(size_t)p];
            const int64_t r0 = row_start[p];
            row_of.assign((size_t)n, -1);
            bool bad = false;
            for (int64_t r = r0; r < r0 + n && !bad; ++r) {
                const int sid = square_id ? square_id[r] : (int)(r - r0);
                if (sid < 0 || sid >= n || row_of[(size_t)sid] >= 0) bad = true;
                else row_of[(size_t)sid] = r;
            }
            if (bad) {
                live[(size_t)p] = 0;
                put(out[p].reason, sizeof out[p].reason,
                    "n=" + std::to_string(n) + ": square_ids should be 0.." + std::to_string(n - 1));
                continue;
            }
            for (int i = 0; i < n; ++i) {
                const int64_t r = row_of[(size_t)i];
                for (int k = 0; k < 3; ++k) {
                    const int64_t a = lit_off[3 * r + k], b = lit_off[3 * r + k + 1];
                    if (b < a) {
                        bad_row[(size_t)t] = r;
                        return;
                    }
                    const size_t q = (size_t)(3 * (pk_sq0[(size_t)p] + i) + k);
                    if (do_rt) {
                        const std::string s2 = roundtrip(text + a, (size_t)(b - a));
                        raw_off[q] = (int64_t)rt[(size_t)t].size();
                        raw_len[q] = (int32_t)s2.size();
                        rt[(size_t)t] += s2;
                    } else {
                        raw_off[q] = a;
                        raw_len[q] = (int32_t)std::min<int64_t>(b - a, 1 << 20);
                    }
                }
            }
        }
    };
    if (nt == 1) {
        slice(0);
    } else {
        std::vector<std::thread> pool;
        for (int t = 0; t < nt; ++t) pool.emplace_back(slice, t);
        for (auto& th : pool) th.join();
    }
    for (int t = 0; t < nt; ++t)
        SQS_REQUIRE(bad_row[(size_t)t] < 0, "literal offsets not monotone at row %lld", (long long)bad_row[(size_t)t]);
    std::string rt_text;  // round-tripped literals, when requested
    if (do_rt) {
        size_t base = 0;
        for (int t = 0; t < nt; ++t) {
            if (base)
                for (int p = p_lo[(size_t)t]; p < p_lo[(size_t)t + 1]; ++p) {
                    if (!live[(size_t)p]) continue;
                    for (int64_t q = 3 * pk_sq0[(size_t)p]; q < 3 * (pk_sq0[(size_t)p] + pk_n[(size_t)p]); ++q)
                        raw_off[(size_t)q] += (int64_t)base;
                }
            base += rt[(size_t)t].size();
        }
        rt_text.reserve(base);
        for (int t = 0; t < nt; ++t) rt_text += rt[(size_t)t];
    }
    const char* blob = do_rt ? rt_text.data() : (h_text ? h_text : text);
    size_t blob_bytes = do_rt ? rt_text.size() : (size_t)lit_off[3 * row_start[count]];
    if (blob_bytes == 0) blob_bytes = 1;
    // buckets by n
    std::vector<int32_t> bk[3];
    for (int p = 0; p < count; ++p) {
        if (!live[(size_t)p]) continue;
        const int n = pk_n[(size_t)p];
        bk[n <= 64 ? 0 : (n <= 256 ? 1 : 2)].push_back(p);
    }
    const uint32_t cap = (uint32_t)std::min<int64_t>(16 * S + 4096, 1ll << 31);
    // device buffers (one staging allocation per call; reused when large enough)
    struct Seg { size_t off, bytes; };
    size_t tot = 0;
    auto seg = [&](size_t bytes) { Seg s{tot, bytes}; tot += (bytes + 255) & ~(size_t)255; return s; };
    const Seg g_text = seg(blob_bytes), g_off = seg(n3 * 8 + 8), g_len = seg(n3 * 4 + 4);
    const Seg g_n = seg((size_t)count * 4), g_s0 = seg((size_t)count * 8);
    const Seg g_b0 = seg(bk[0].size() * 4 + 4), g_b1 = seg(bk[1].size() * 4 + 4), g_b2 = seg(bk[2].size() * 4 + 4);
    const Seg g_lits = seg((size_t)(3 * S + 3) * sizeof(Lit)), g_out = seg((size_t)count * sizeof(PkOut));
    const Seg g_pa = seg((size_t)cap * sizeof(Pair)), g_pb = seg((size_t)cap * sizeof(Pair)), g_cnt = seg(64);
    const Seg g_slot = seg((size_t)S * sizeof(int32_t) + 4), g_list = seg((size_t)S * sizeof(SqRef) + 8);
    if (int r = ctx->d_misc.reserve(tot)) return r;
    char* D = (char*)ctx->d_misc.p;
    auto up = [&](const Seg& s, const void* h, size_t bytes) -> int {
        if (bytes) SQS_CUDA(cudaMemcpyAsync(D + s.off, h, bytes, cudaMemcpyHostToDevice, ctx->stream));
        return SQS_OK;
    };
    if (int r = up(g_text, blob, do_rt ? rt_text.size() : (size_t)lit_off[3 * row_start[count]])) return r;
    if (int r = up(g_off, raw_off, n3 * 8)) return r;
    if (int r = up(g_len, raw_len, n3 * 4)) return r;
    if (int r = up(g_n, pk_n.data(), (size_t)count * 4)) return r;
    if (int r = up(g_s0, pk_sq0.data(), (size_t)count * 8)) return r;
    if (int r = up(g_b0, bk[0].data(), bk[0].size() * 4)) return r;
    if (int r = up(g_b1, bk[1].data(), bk[1].size() * 4)) return r;
    if (int r = up(g_b2, bk[2].data(), bk[2].size() * 4)) return r;
    SQS_CUDA(cudaMemsetAsync(D + g_out.off, 0, g_out.bytes, ctx->stream));
    SQS_CUDA(cudaMemsetAsync(D + g_cnt.off, 0, 64, ctx->stream));
    PkOut* d_out = (PkOut*)(D + g_out.off);
    Pair* pa = (Pair*)(D + g_pa.off);
    Pair* pb = (Pair*)(D + g_pb.off);
    uint32_t* cnt = (uint32_t*)(D + g_cnt.off);
    const char* d_text = D + g_text.off;
    const int64_t* d_off = (const int64_t*)(D + g_off.off);
    const int32_t* d_len = (const int32_t*)(D + g_len.off);
    const int32_t* d_n = (const int32_t*)(D + g_n.off);
    const int64_t* d_s0 = (const int64_t*)(D + g_s0.off);
    Lit* d_lits = (Lit*)(D + g_lits.off);
    if (int r = launch_packing<64, 64>(ctx, (int)bk[0].size(), (const int32_t*)(D + g_b0.off), d_n, d_s0, d_text,
                                       d_off, d_len, d_lits, d_out, pa, cnt, cap)) return r;
    if (int r = launch_packing<128, 256>(ctx, (int)bk[1].size(), (const int32_t*)(D + g_b1.off), d_n, d_s0, d_text,
                                         d_off, d_len, d_lits, d_out, pa, cnt, cap)) return r;
    if (int r = launch_packing<256, 1024>(ctx, (int)bk[2].size(), (const int32_t*)(D + g_b2.off), d_n, d_s0,
                                          d_text, d_off, d_len, d_lits, d_out, pa, cnt, cap)) return r;
    int32_t* slot_of = (int32_t*)(D + g_slot.off);
    SqRef* list = (SqRef*)(D + g_list.off);
    // FP64 prefilter pa -> pb, then the 7-, 15- and 58-limb stages pb -> pa -> pb
    if (int r = launch_fp64(ctx, pa, cnt, cap, pb, cnt + 5, cap, d_s0, d_lits, d_text, d_out, ctx->sm_count * 8))
        return r;
    if (int r = cached_stage<7>(ctx, pb, cnt + 5, cap, pa, cnt + 1, d_s0, d_lits, d_text, d_out, slot_of, list, cnt + 3,
                                S))
        return r;
    if (int r = cached_stage<15>(ctx, pa, cnt + 1, cap, pb, cnt + 2, d_s0, d_lits, d_text, d_out, slot_of, list,
                                 cnt + 3, S))
        return r;
    if (int r = cached_stage<58>(ctx, pb, cnt + 2, cap, nullptr, nullptr, d_s0, d_lits, d_text, d_out, slot_of, list,
                                 cnt + 3, S))
        return r;
    std::vector<PkOut> h((size_t)count);
    SQS_CUDA(cudaMemcpyAsync(h.data(), d_out, (size_t)count * sizeof(PkOut), cudaMemcpyDeviceToHost, ctx->stream));
    SQS_CUDA(cudaStreamSynchronize(ctx->stream));
    for (int p = 0; p < count; ++p) {
        if (!live[(size_t)p]) continue;
        sqs_verdict& v = out[p];
        const PkOut& o = h[(size_t)p];
        const int n = pk_n[(size_t)p];
        const std::string N = std::to_string(n);
        if (o.flags & kPairOverflow) {
            set_error("packing %d: undecided-pair list overflowed", p);
            return SQS_ENOMEM;
        }
        if (o.err_key != kNoKey) {
            static const char* what[4] = {"cannot parse coordinates", "value out of range for a double",
                                          "coordinate out of bounds", "angle out of bounds"};
            put(v.reason, sizeof v.reason,
                "n=" + N + ", square " + std::to_string(o.err_key / 4) + ": " + what[o.err_key % 4]);
            continue;
        }
        if (o.fkey != kNoPair) {
            put(v.reason, sizeof v.reason,
                "infeasible: Squares " + std::to_string(o.fu) + " and " + std::to_string(o.fv) +
                    " overlap (float check)");
            continue;
        }
        if (o.flags & kCertOverlap) {
            put(v.reason, sizeof v.reason, "infeasible: Squares overlap (certified)");
            continue;
        }
        if (o.flags & kUndecidable) {
            put(v.reason, sizeof v.reason, "infeasible: Overlap undecidable at max precision");
            continue;
        }
        const double sf = fx::approx(o.side), lb = std::sqrt((double)n);
        if (sf < lb - 1e-7) {
            put(v.reason, sizeof v.reason, "infeasible: L is below area lower bound");
            continue;
        }
        v.ok = 1;
        put(v.reason, sizeof v.reason, "ok");
        put(v.L, sizeof v.L, fifty(o.side));
        v.score = std::max(0.0, sf / lb - 1.0);
    }
    return SQS_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free certification: the same kernels, with every device buffer
// carved from one file-scope array and every host buffer static.  For callers
// that must not allocate device memory at run time -- a host that owns all
// GPU memory through its own pool, a real-time loop that forbids allocation
// after start-up -- at the price of fixed limits and of a process-wide
// buffer that concurrent calls share.
namespace sqs {
namespace cert {

constexpr int kStaticMaxSquares = 16384;
constexpr int kStaticMaxPackings = 4096;
constexpr size_t kStaticMaxText = 2u << 20;               // literal bytes per call
constexpr uint32_t kStaticPairCap = 16u * kStaticMaxSquares + 4096u;

constexpr size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }
constexpr size_t kSoText = 0;
constexpr size_t kSoOff = kSoText + al256(kStaticMaxText);
constexpr size_t kSoLen = kSoOff + al256(sizeof(int64_t) * 3 * kStaticMaxSquares);
constexpr size_t kSoN = kSoLen + al256(sizeof(int32_t) * 3 * kStaticMaxSquares);
constexpr size_t kSoS0 = kSoN + al256(sizeof(int32_t) * kStaticMaxPackings);
constexpr size_t kSoBk = kSoS0 + al256(sizeof(int64_t) * kStaticMaxPackings);
constexpr size_t kSoLits = kSoBk + al256(sizeof(int32_t) * kStaticMaxPackings);
constexpr size_t kSoOut = kSoLits + al256(sizeof(Lit) * 3 * kStaticMaxSquares);
constexpr size_t kSoPa = kSoOut + al256(sizeof(PkOut) * kStaticMaxPackings);
constexpr size_t kSoPb = kSoPa + al256(sizeof(Pair) * kStaticPairCap);
constexpr size_t kSoCnt = kSoPb + al256(sizeof(Pair) * kStaticPairCap);
constexpr size_t kStaticScratchBytes = kSoCnt + 256;  // about 7.6 MiB

// The scratch every call of sqs_certify_batch_static shares.  In host code
// this name is only a stand-in: the device address comes from
// cudaGetSymbolAddress, taken once per device.
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];
static void* s_scratch_addr[64] = {nullptr};
static std::atomic<bool> s_ready[64];
static std::mutex s_setup_mu;
// Set while a call runs: the scratch and the host staging below are shared
// by every call in the process, so a call that would overlap another is
// refused instead of racing with it.
static std::atomic_flag s_busy = ATOMIC_FLAG_INIT;

// Host staging (static, not heap): literal slices in square-id order, packing
// tables, round-tripped literals, the per-packing records read back.
static int64_t s_raw_off[3 * kStaticMaxSquares];
static int32_t s_raw_len[3 * kStaticMaxSquares];
static int32_t s_pk_n[kStaticMaxPackings];
static int64_t s_pk_sq0[kStaticMaxPackings];
static int32_t s_bucket[kStaticMaxPackings];
static unsigned char s_live[kStaticMaxPackings];
static int64_t s_row_of[kMaxN];
static char s_rt_text[kStaticMaxText];
static char s_lit_tmp[4096];
static PkOut s_out[kStaticMaxPackings];

// Per-device set-up of the allocation-free path, once, with that device
// current: the device address of the static array (cudaGetSymbolAddress;
// under lazy module loading this is also what loads the module holding the
// array), the certifier's constants, and one launch of each stage kernel
// with nothing to do, which loads the kernels and lets the driver size the
// local memory their stacks need.  Everything a later call uses is then in
// place, so later calls allocate nothing.
template <int T, int NMAX>
static int packing_attr() {
    const size_t smem = (size_t)NMAX * (sizeof(FSq) + 5 * sizeof(double) + sizeof(int16_t));
    SQS_CUDA(cudaFuncSetAttribute(cert_packing_kernel<T, NMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    return SQS_OK;
}

static int static_setup(sqs_ctx* ctx) {
    const int dev = ctx->device & 63;
    if (s_ready[dev]) return SQS_OK;
    std::lock_guard<std::mutex> lk(s_setup_mu);
    if (s_ready[dev]) return SQS_OK;
    void* p = nullptr;
    SQS_CUDA(cudaGetSymbolAddress(&p, g_static_scratch));
    if (int r = upload_consts(ctx->device)) return r;
    if (int r = packing_attr<64, 64>()) return r;
    if (int r = packing_attr<128, 256>()) return r;
    if (int r = packing_attr<256, 1024>()) return r;
    char* D = (char*)p;
    Pair* pa = (Pair*)(D + kSoPa);
    uint32_t* cnt = (uint32_t*)(D + kSoCnt);
    SQS_CUDA(cudaMemsetAsync(cnt, 0, 64, ctx->stream));
    const int64_t* d_s0 = (const int64_t*)(D + kSoS0);
    const Lit* d_lits = (const Lit*)(D + kSoLits);
    PkOut* d_out = (PkOut*)(D + kSoOut);
    if (int r = launch_fp64(ctx, pa, cnt, 0, nullptr, nullptr, 0, d_s0, d_lits, D, d_out, 1)) return r;
    if (int r = launch_stage<7>(ctx, pa, cnt, 0, nullptr, nullptr, 0, d_s0, d_lits, D, d_out, 1)) return r;
    if (int r = launch_stage<15>(ctx, pa, cnt, 0, nullptr, nullptr, 0, d_s0, d_lits, D, d_out, 1)) return r;
    if (int r = launch_stage<58>(ctx, pa, cnt, 0, nullptr, nullptr, 0, d_s0, d_lits, D, d_out, 1)) return r;
    SQS_CUDA(cudaStreamSynchronize(ctx->stream));
    s_scratch_addr[dev] = p;
    s_ready[dev] = true;
    return SQS_OK;
}

namespace {
struct BusyGuard {
    bool held;
    BusyGuard() : held(!s_busy.test_and_set(std::memory_order_acquire)) {}
    ~BusyGuard() {
        if (held) s_busy.clear(std::memory_order_release);
    }
};
}  // namespace

}  // namespace cert
}  // namespace sqs

extern "C" int sqs_certify_batch_static(sqs_ctx* ctx, int count, const int32_t* n_of, const int64_t* row_start,
                                        const int32_t* square_id, const char* text, const int64_t* lit_off,
                                        int flags, sqs_verdict* out) {
    if (int r = enter(ctx)) return r;
    BusyGuard busy;
    if (!busy.held) {
        set_error("sqs_certify_batch_static: another call is in progress (all calls share one static scratch "
                  "array and must not overlap)");
        return SQS_EBUSY;
    }
    SQS_REQUIRE(count >= 0 && count <= kStaticMaxPackings, "count %d out of 0..%d (static certifier limit)", count,
                kStaticMaxPackings);
    // the first call on a device (count == 0 does only this) sets the path up
    if (int r = static_setup(ctx)) return r;
    if (count == 0) return SQS_OK;
    SQS_REQUIRE(n_of && row_start && text && lit_off && out, "null host pointer");
    const int dev = ctx->device & 63;
    const bool do_rt = (flags & SQS_CERT_ROUNDTRIP) != 0;
    // envelope checks and literal slices, as sqs_certify_batch does them
    int64_t S = 0;
    size_t rt_used = 0;
    for (int p = 0; p < count; ++p) {
        const int n = n_of[p];
        sqs_verdict& v = out[p];
        std::memset(&v, 0, sizeof v);
        v.n = n;
        s_live[p] = 0;
        SQS_REQUIRE(n >= 1 && n <= kMaxN, "packing %d: n=%d out of 1..%d", p, n, kMaxN);
        v.score = grid_score(n);
        const int64_t r0 = row_start[p], r1 = row_start[p + 1];
        SQS_REQUIRE(r1 >= r0, "packing %d: row_start not monotone", p);
        if (r1 - r0 != n) {
            std::snprintf(v.reason, sizeof v.reason, "n=%d: expected %d rows, got %lld", n, n, (long long)(r1 - r0));
            continue;
        }
        for (int i = 0; i < n; ++i) s_row_of[i] = -1;
        bool bad = false;
        for (int64_t r = r0; r < r1 && !bad; ++r) {
            const int sid = square_id ? square_id[r] : (int)(r - r0);
            if (sid < 0 || sid >= n || s_row_of[sid] >= 0) bad = true;
            else s_row_of[sid] = r;
        }
        if (bad) {
            std::snprintf(v.reason, sizeof v.reason, "n=%d: square_ids should be 0..%d", n, n - 1);
            continue;
        }
        SQS_REQUIRE(S + n <= kStaticMaxSquares, "more than %d squares in one static-certifier call",
                    kStaticMaxSquares);
        s_live[p] = 1;
        s_pk_n[p] = n;
        s_pk_sq0[p] = S;
        for (int i = 0; i < n; ++i) {
            const int64_t r = s_row_of[i];
            for (int k = 0; k < 3; ++k) {
                const int64_t a = lit_off[3 * r + k], b = lit_off[3 * r + k + 1];
                SQS_REQUIRE(b >= a, "literal offsets not monotone at row %lld", (long long)r);
                const int64_t q = 3 * (S + i) + k;
                if (do_rt) {
                    SQS_REQUIRE((size_t)(b - a) < sizeof(s_lit_tmp), "literal longer than %zu bytes",
                                sizeof(s_lit_tmp) - 1);
                    std::memcpy(s_lit_tmp, text + a, (size_t)(b - a));
                    s_lit_tmp[b - a] = 0;
                    char buf[40];
                    const size_t len = roundtrip_into(std::strtod(s_lit_tmp, nullptr), buf);
                    SQS_REQUIRE(rt_used + len <= kStaticMaxText, "literals exceed %zu bytes", kStaticMaxText);
                    std::memcpy(s_rt_text + rt_used, buf, len);
                    s_raw_off[q] = (int64_t)rt_used;
                    s_raw_len[q] = (int32_t)len;
                    rt_used += len;
                } else {
                    s_raw_off[q] = a;
                    s_raw_len[q] = (int32_t)std::min<int64_t>(b - a, 1 << 20);
                }
            }
        }
        S += n;
    }
    const size_t text_bytes = do_rt ? rt_used : (size_t)lit_off[3 * row_start[count]];
    SQS_REQUIRE(text_bytes <= kStaticMaxText, "literals exceed %zu bytes (static certifier limit)", kStaticMaxText);
    int nb[3] = {0, 0, 0};
    for (int p = 0; p < count; ++p)
        if (s_live[p]) ++nb[s_pk_n[p] <= 64 ? 0 : (s_pk_n[p] <= 256 ? 1 : 2)];
    int fill[3] = {0, nb[0], nb[0] + nb[1]};
    for (int p = 0; p < count; ++p) {
        if (!s_live[p]) continue;
        const int b = s_pk_n[p] <= 64 ? 0 : (s_pk_n[p] <= 256 ? 1 : 2);
        s_bucket[fill[b]++] = p;
    }
    char* D = (char*)s_scratch_addr[dev];
    cudaStream_t st = ctx->stream;
    if (text_bytes)
        SQS_CUDA(cudaMemcpyAsync(D + kSoText, do_rt ? s_rt_text : text, text_bytes, cudaMemcpyHostToDevice, st));
    SQS_CUDA(cudaMemcpyAsync(D + kSoOff, s_raw_off, sizeof(int64_t) * 3 * (size_t)S, cudaMemcpyHostToDevice, st));
    SQS_CUDA(cudaMemcpyAsync(D + kSoLen, s_raw_len, sizeof(int32_t) * 3 * (size_t)S, cudaMemcpyHostToDevice, st));
    SQS_CUDA(cudaMemcpyAsync(D + kSoN, s_pk_n, sizeof(int32_t) * (size_t)count, cudaMemcpyHostToDevice, st));
    SQS_CUDA(cudaMemcpyAsync(D + kSoS0, s_pk_sq0, sizeof(int64_t) * (size_t)count, cudaMemcpyHostToDevice, st));
    SQS_CUDA(cudaMemcpyAsync(D + kSoBk, s_bucket, sizeof(int32_t) * (size_t)(nb[0] + nb[1] + nb[2]),
                             cudaMemcpyHostToDevice, st));
    // the shared scratch keeps the previous call's contents: clear what starts at zero
    SQS_CUDA(cudaMemsetAsync(D + kSoOut, 0, sizeof(PkOut) * (size_t)count, st));
    SQS_CUDA(cudaMemsetAsync(D + kSoCnt, 0, 64, st));
    const char* d_text = D + kSoText;
    const int64_t* d_off = (const int64_t*)(D + kSoOff);
    const int32_t* d_len = (const int32_t*)(D + kSoLen);
    const int32_t* d_n = (const int32_t*)(D + kSoN);
    const int64_t* d_s0 = (const int64_t*)(D + kSoS0);
    const int32_t* d_bk = (const int32_t*)(D + kSoBk);
    Lit* d_lits = (Lit*)(D + kSoLits);
    PkOut* d_out = (PkOut*)(D + kSoOut);
    Pair* pa = (Pair*)(D + kSoPa);
    Pair* pb = (Pair*)(D + kSoPb);
    uint32_t* cnt = (uint32_t*)(D + kSoCnt);
    const uint32_t cap = kStaticPairCap;
    if (int r = launch_packing<64, 64>(ctx, nb[0], d_bk, d_n, d_s0, d_text, d_off, d_len, d_lits, d_out, pa, cnt, cap))
        return r;
    if (int r = launch_packing<128, 256>(ctx, nb[1], d_bk + nb[0], d_n, d_s0, d_text, d_off, d_len, d_lits, d_out,
                                         pa, cnt, cap))
        return r;
    if (int r = launch_packing<256, 1024>(ctx, nb[2], d_bk + nb[0] + nb[1], d_n, d_s0, d_text, d_off, d_len, d_lits,
                                          d_out, pa, cnt, cap))
        return r;
    const int blocks = ctx->sm_count * 8;
    if (int r = launch_fp64(ctx, pa, cnt, cap, pb, cnt + 5, cap, d_s0, d_lits, d_text, d_out, blocks)) return r;
    if (int r = launch_stage<7>(ctx, pb, cnt + 5, cap, pa, cnt + 1, cap, d_s0, d_lits, d_text, d_out, blocks)) return r;
    if (int r = launch_stage<15>(ctx, pa, cnt + 1, cap, pb, cnt + 2, cap, d_s0, d_lits, d_text, d_out, blocks))
        return r;
    if (int r = launch_stage<58>(ctx, pb, cnt + 2, cap, nullptr, nullptr, 0, d_s0, d_lits, d_text, d_out, blocks))
        return r;
    SQS_CUDA(cudaMemcpyAsync(s_out, d_out, sizeof(PkOut) * (size_t)count, cudaMemcpyDeviceToHost, st));
    SQS_CUDA(cudaStreamSynchronize(st));
    static const char* what[4] = {"cannot parse coordinates", "value out of range for a double",
                                  "coordinate out of bounds", "angle out of bounds"};
    for (int p = 0; p < count; ++p) {
        if (!s_live[p]) continue;
        sqs_verdict& v = out[p];
        const PkOut& o = s_out[p];
        const int n = s_pk_n[p];
        if (o.flags & kPairOverflow) {
            set_error("packing %d: undecided-pair list overflowed", p);
            return SQS_ENOMEM;
        }
        if (o.err_key != kNoKey) {
            std::snprintf(v.reason, sizeof v.reason, "n=%d, square %u: %s", n, o.err_key / 4, what[o.err_key % 4]);
            continue;
        }
        if (o.fkey != kNoPair) {
            std::snprintf(v.reason, sizeof v.reason, "infeasible: Squares %d and %d overlap (float check)", o.fu, o.fv);
            continue;
        }
        if (o.flags & kCertOverlap) {
            std::snprintf(v.reason, sizeof v.reason, "infeasible: Squares overlap (certified)");
            continue;
        }
        if (o.flags & kUndecidable) {
            std::snprintf(v.reason, sizeof v.reason, "infeasible: Overlap undecidable at max precision");
            continue;
        }
        const double sf = fx::approx(o.side), lb = std::sqrt((double)n);
        if (sf < lb - 1e-7) {
            std::snprintf(v.reason, sizeof v.reason, "infeasible: L is below area lower bound");
            continue;
        }
        v.ok = 1;
        std::snprintf(v.reason, sizeof v.reason, "ok");
        fifty_into(o.side, v.L, sizeof v.L);
        v.score = std::max(0.0, sf / lb - 1.0);
    }
    return SQS_OK;
}
