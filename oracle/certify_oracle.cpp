// TEST INFRASTRUCTURE ONLY -- the CPU oracle for the interval certifier.
//
// Loaded only by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
// leg, as the checker of the CUDA certifier; nothing in the product links it.
//
// A single-threaded C++ restatement of the reference certifier's algorithm
// (cuda/certifier.cpp), which itself mirrors the Kaggle v20 metric:
//   fixed-point numbers, base 1e9, FL fractional limbs   certifier.cpp:32-105
//   add / sub / 1-ulp / mul with rounding / small div   :107-235
//   intervals                                            :237-263
//   decimal parse (truncating / directed) + dyadic test  :265-394
//   Taylor sin/cos, point and interval                   :413-503
//   literal validation                                   :505-529
//   float corners, AABB, float SAT prefilter             :543-588
//   interval corner cache + interval SAT                 :590-703
//   escalation stage                                     :705-724
//   evaluate one packing (checks, Fix<9> L, sweep,
//     escalation 7 -> 15 -> 58, area bound, L string)    :738-912
//   pandas round-trip emulation of one literal           :914-929
// Parity is pinned against the reference certifier compiled into oracle/_ref
// and against L strings produced by the reference's Python metric.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

namespace orc {

constexpr uint64_t B9 = 1000000000ULL;

template <int F>
struct Fx {
    int neg = 0;                 // 1 when negative; zero is always non-negative
    uint64_t d[F + 1] = {0};     // d[0] integer limb, d[1..F] fraction limbs

    bool zero() const {
        for (int i = 0; i <= F; ++i)
            if (d[i]) return false;
        return true;
    }
    void fix_zero() {
        if (zero()) neg = 0;
    }
    static Fx of(long long v) {
        Fx r;
        if (v < 0) { r.neg = 1; v = -v; }
        r.d[0] = (uint64_t)v;
        return r;
    }
    double approx() const {
        double v = (double)d[0], sc = 1.0;
        for (int i = 1; i <= std::min(F, 4); ++i) {
            sc *= 1e-9;
            v += (double)d[i] * sc;
        }
        return neg ? -v : v;
    }
};

template <int F>
int mag_cmp(const Fx<F>& a, const Fx<F>& b) {
    for (int i = 0; i <= F; ++i)
        if (a.d[i] != b.d[i]) return a.d[i] < b.d[i] ? -1 : 1;
    return 0;
}

template <int F>
int cmp(const Fx<F>& a, const Fx<F>& b) {
    if (a.zero() && b.zero()) return 0;
    if (a.neg != b.neg) return a.neg ? -1 : 1;
    int c = mag_cmp(a, b);
    return a.neg ? -c : c;
}

template <int F>
Fx<F> mag_add(const Fx<F>& a, const Fx<F>& b, int neg) {
    Fx<F> r;
    r.neg = neg;
    uint64_t c = 0;
    for (int i = F; i >= 1; --i) {
        uint64_t s = a.d[i] + b.d[i] + c;
        c = s >= B9;
        r.d[i] = c ? s - B9 : s;
    }
    r.d[0] = a.d[0] + b.d[0] + c;
    r.fix_zero();
    return r;
}

template <int F>
Fx<F> mag_sub(const Fx<F>& a, const Fx<F>& b, int neg) {  // |a| >= |b|
    Fx<F> r;
    r.neg = neg;
    int64_t br = 0;
    for (int i = F; i >= 1; --i) {
        int64_t s = (int64_t)a.d[i] - (int64_t)b.d[i] - br;
        br = s < 0;
        r.d[i] = (uint64_t)(br ? s + (int64_t)B9 : s);
    }
    r.d[0] = (uint64_t)((int64_t)a.d[0] - (int64_t)b.d[0] - br);
    r.fix_zero();
    return r;
}

template <int F>
Fx<F> add(const Fx<F>& a, const Fx<F>& b) {
    if (a.neg == b.neg) return mag_add(a, b, a.neg);
    int c = mag_cmp(a, b);
    if (c == 0) return Fx<F>();
    return c > 0 ? mag_sub(a, b, a.neg) : mag_sub(b, a, b.neg);
}

template <int F>
Fx<F> neg(Fx<F> a) {
    a.neg = !a.neg;
    a.fix_zero();
    return a;
}

template <int F>
Fx<F> sub(const Fx<F>& a, const Fx<F>& b) { return add(a, neg(b)); }

template <int F>
void bump(Fx<F>& a) {  // |a| += one unit of the last limb
    for (int i = F; i >= 1; --i) {
        if (++a.d[i] < B9) return;
        a.d[i] = 0;
    }
    a.d[0] += 1;
}

// rnd: 0 = round half up on the first dropped limb, -1 toward -inf, +1 toward +inf.
template <int F>
Fx<F> mul(const Fx<F>& a, const Fx<F>& b, int rnd) {
    if (a.zero() || b.zero()) return Fx<F>();
    uint64_t p[2 * F + 2] = {0};
    for (int i = 0; i <= F; ++i) {
        if (!a.d[i]) continue;
        uint64_t c = 0;
        for (int j = F; j >= 0; --j) {
            unsigned __int128 t = (unsigned __int128)p[i + j] + (unsigned __int128)a.d[i] * b.d[j] + c;
            p[i + j] = (uint64_t)(t % B9);
            c = (uint64_t)(t / B9);
        }
        for (int k = i - 1; c && k >= 0; --k) {  // carry out of limb 0 is dropped
            uint64_t s = p[k] + c;
            p[k] = s % B9;
            c = s / B9;
        }
    }
    Fx<F> r;
    r.neg = a.neg ^ b.neg;
    for (int i = 0; i <= F; ++i) r.d[i] = p[i];
    bool tail = false;
    for (int i = F + 1; i <= 2 * F; ++i) tail |= p[i] != 0;
    if (rnd == 0) {
        if (p[F + 1] >= B9 / 2) bump(r);
    } else if (tail && ((rnd > 0) == !r.neg)) {
        bump(r);
    }
    r.fix_zero();
    return r;
}

template <int F>
Fx<F> div_u(const Fx<F>& a, uint64_t den) {  // round half up on the remainder
    Fx<F> r;
    r.neg = a.neg;
    uint64_t rem = 0;
    for (int i = 0; i <= F; ++i) {
        unsigned __int128 t = (unsigned __int128)rem * B9 + a.d[i];
        r.d[i] = (uint64_t)(t / den);
        rem = (uint64_t)(t % den);
    }
    if (rem * 2 >= den) bump(r);
    r.fix_zero();
    return r;
}

template <int F>
struct Iv {
    Fx<F> lo, hi;
};

template <int F>
Iv<F> iadd(const Iv<F>& a, const Iv<F>& b) { return {add(a.lo, b.lo), add(a.hi, b.hi)}; }
template <int F>
Iv<F> isub(const Iv<F>& a, const Iv<F>& b) { return {sub(a.lo, b.hi), sub(a.hi, b.lo)}; }
template <int F>
Iv<F> ineg(const Iv<F>& a) { return {neg(a.hi), neg(a.lo)}; }
template <int F>
Iv<F> imul(const Iv<F>& a, const Iv<F>& b) {
    const Fx<F>* x[2] = {&a.lo, &a.hi};
    const Fx<F>* y[2] = {&b.lo, &b.hi};
    Fx<F> lo = mul(*x[0], *y[0], -1), hi = mul(*x[0], *y[0], +1);
    for (int k = 1; k < 4; ++k) {
        Fx<F> dn = mul(*x[k >> 1], *y[k & 1], -1), up = mul(*x[k >> 1], *y[k & 1], +1);
        if (cmp(dn, lo) < 0) lo = dn;
        if (cmp(up, hi) > 0) hi = up;
    }
    return {lo, hi};
}

// Decimal literal split into its digit string and decimal exponent.
struct Lit {
    std::string digits;  // all mantissa digits, no dot
    long long point;     // number of digits before the decimal point (may be <0 or > size)
    int negative;
};

static Lit split(const std::string& s) {
    size_t i = 0, e = s.size();
    while (i < e && isspace((unsigned char)s[i])) ++i;
    while (e > i && isspace((unsigned char)s[e - 1])) --e;
    Lit L{{}, 0, 0};
    if (i < e && (s[i] == '+' || s[i] == '-')) L.negative = s[i++] == '-';
    long long frac = 0;
    bool dot = false;
    for (; i < e && s[i] != 'e' && s[i] != 'E'; ++i) {
        if (s[i] == '.') dot = true;
        else { L.digits.push_back(s[i]); frac += dot; }
    }
    long long ex = 0;
    if (i < e) {
        ++i;
        int es = 1;
        if (i < e && (s[i] == '+' || s[i] == '-')) es = s[i++] == '-' ? -1 : 1;
        for (; i < e && isdigit((unsigned char)s[i]); ++i) ex = ex * 10 + (s[i] - '0');
        ex *= es;
    }
    L.point = (long long)L.digits.size() - frac + ex;
    return L;
}

static inline int digit_at(const Lit& L, long long pos) {
    return (pos >= 0 && pos < (long long)L.digits.size()) ? L.digits[(size_t)pos] - '0' : 0;
}

// rnd 0 truncates; -1 / +1 round the magnitude away from zero in that direction
// when any digit beyond the last limb is non-zero.
template <int F>
Fx<F> parse(const std::string& s, int rnd) {
    Lit L = split(s);
    Fx<F> r;
    r.neg = L.negative;
    uint64_t iv = 0;
    for (long long k = 0; k < L.point; ++k) iv = iv * 10 + (uint64_t)digit_at(L, k);
    r.d[0] = iv;
    for (int l = 1; l <= F; ++l) {
        uint64_t v = 0;
        for (int k = 0; k < 9; ++k) v = v * 10 + (uint64_t)digit_at(L, L.point + (long long)(l - 1) * 9 + k);
        r.d[l] = v;
    }
    bool tail = false;
    for (long long pos = std::max(0LL, L.point + 9LL * F); pos < (long long)L.digits.size() && !tail; ++pos)
        tail = L.digits[(size_t)pos] != '0';
    if (tail && rnd != 0 && ((rnd > 0) == !L.negative)) bump(r);
    r.fix_zero();
    return r;
}

// True when the literal's value has a finite binary expansion, decided for at
// most 25 effective decimal places (more is treated as non-dyadic).
static bool dyadic(const std::string& s) {
    Lit L = split(s);
    std::string dg = L.digits;
    long long places = (long long)dg.size() - L.point;
    while (places > 0 && !dg.empty() && dg.back() == '0') { dg.pop_back(); --places; }
    if (places <= 0) return true;
    if (places > 25) return false;
    for (long long k = 0; k < places; ++k) {
        if (dg.empty()) return true;
        if ((dg.back() - '0') % 5) return false;
        std::string q;
        int rem = 0;
        for (char ch : dg) {
            int cur = rem * 10 + (ch - '0');
            if (!q.empty() || cur / 5) q.push_back((char)('0' + cur / 5));
            rem = cur % 5;
        }
        dg.swap(q);
    }
    return true;
}

template <int F>
Iv<F> parse_iv(const std::string& s) {
    Iv<F> r{parse<F>(s, -1), parse<F>(s, +1)};
    if (!dyadic(s)) {
        Fx<F> u;
        u.d[F] = 1;
        r.lo = sub(r.lo, u);
        r.hi = add(r.hi, u);
    }
    return r;
}

static const char* kHalfPi =
    "1.5707963267948966192313216916397514420985846996875529104874722961539082031431044993140174126710585339"
    "9107404325664115332354692230477529111586267970406424055872514205135096926055277982231147447746519098"
    "2214405487832966723064237824116893391582635600954572824283161565386415559563044484210977355059400485"
    "7492389293099245510655716316154220989218499846888949675083019800051100514872368941154883214599416258"
    "7630228031340772652010253145121415210968393898212262598912242342639728019727481121132833606270987663"
    "3184560871636462872546121833290233099787539786414835847812261143213250625359595866490484368352035968";
static const char* kTwoPi =
    "6.2831853071795864769252867665590057683943387987502116419498891846156328125724179972560696506842341359"
    "6429617302656461329418768921910116446345071881625696223490056820540387704221111928924589790986076392"
    "8857621951331866892256951296467573566330542403818291297132646261545662238252177936843909420237601942"
    "9969557172396982042622865264616883956873999387555798700332079200204402059489475764619532858397665035"
    "0520912125363090608041012580485660843873575592848905039564896937055891207890992448453133442508395065"
    "2738243486545851490184487333160932399150159145659343391249044572853002501438383465961937473408143872";

// Taylor sums of sin and cos at x (|x| <= pi/4) with round-half-up limbs.
template <int F>
void taylor(const Fx<F>& x, Fx<F>& sn, Fx<F>& cs, int terms) {
    Fx<F> x2 = mul(x, x, 0);
    Fx<F> ct = Fx<F>::of(1), st = x;
    cs = Fx<F>::of(1);
    sn = x;
    for (int m = 1; m <= terms; ++m) {
        ct = div_u(mul(ct, x2, 0), (uint64_t)(2 * m - 1) * (uint64_t)(2 * m));
        ct.neg = (m & 1);
        ct.fix_zero();
        cs = add(cs, ct);
        st = div_u(mul(st, x2, 0), (uint64_t)(2 * m) * (uint64_t)(2 * m + 1));
        st.neg = (m & 1) ? !x.neg : x.neg;
        st.fix_zero();
        sn = add(sn, st);
        if (ct.zero() && st.zero()) break;
    }
}

// Point sin/cos: quadrant from the double approximation, then Taylor.
template <int F>
void sincos_point(const Fx<F>& a, Fx<F>& sn, Fx<F>& cs) {
    static const Fx<F> hp = parse<F>(kHalfPi, 0);
    long long q = (long long)std::round(a.approx() / 1.57079632679489661923);
    Fx<F> r = sub(a, mul(Fx<F>::of(q), hp, 0));
    Fx<F> s0, c0;
    taylor(r, s0, c0, F <= 10 ? 32 : 115);
    switch ((int)((q % 4 + 4) % 4)) {
        case 0: sn = s0; cs = c0; break;
        case 1: sn = c0; cs = neg(s0); break;
        case 2: sn = neg(s0); cs = neg(c0); break;
        default: sn = neg(c0); cs = s0; break;
    }
}

// Interval sin/cos: Taylor at both reduced endpoints, hull widened by one ulp.
template <int F>
void sincos_iv(const Iv<F>& a, Iv<F>& sn, Iv<F>& cs) {
    if (a.lo.zero() && a.hi.zero()) {
        sn = {Fx<F>(), Fx<F>()};
        cs = {Fx<F>::of(1), Fx<F>::of(1)};
        return;
    }
    static const Iv<F> hp = parse_iv<F>(kHalfPi);
    double mid = 0.5 * (a.lo.approx() + a.hi.approx());
    long long q = (long long)std::round(mid / 1.57079632679489661923);
    Fx<F> qf = Fx<F>::of(q);
    Iv<F> r = isub(a, imul(Iv<F>{qf, qf}, hp));
    int terms = F <= 8 ? 28 : (F <= 15 ? 45 : 145);
    Fx<F> sl, cl, sh, ch;
    taylor(r.lo, sl, cl, terms);
    if (cmp(r.lo, r.hi) == 0) { sh = sl; ch = cl; }
    else taylor(r.hi, sh, ch, terms);
    auto hull = [](const Fx<F>& u, const Fx<F>& v, bool peak) {
        Fx<F> lo = cmp(u, v) < 0 ? u : v, hi = cmp(u, v) > 0 ? u : v, e;
        e.d[F] = 1;
        lo = sub(lo, e);
        hi = add(hi, e);
        if (peak && cmp(hi, Fx<F>::of(1)) < 0) hi = Fx<F>::of(1);
        return Iv<F>{lo, hi};
    };
    bool through0 = (r.lo.neg && !r.hi.neg && !r.hi.zero()) || r.lo.zero() || r.hi.zero();
    Iv<F> s0 = hull(sl, sh, false), c0 = hull(cl, ch, through0);
    switch ((int)((q % 4 + 4) % 4)) {
        case 0: sn = s0; cs = c0; break;
        case 1: sn = c0; cs = ineg(s0); break;
        case 2: sn = ineg(s0); cs = ineg(c0); break;
        default: sn = ineg(c0); cs = s0; break;
    }
}

static bool literal_ok(const std::string& raw, std::string& out) {
    size_t a = 0, b = raw.size();
    while (a < b && isspace((unsigned char)raw[a])) ++a;
    while (b > a && isspace((unsigned char)raw[b - 1])) --b;
    out = raw.substr(a, b - a);
    if (out.empty() || out.size() > 100) return false;
    size_t i = 0, n = out.size();
    if (out[i] == '+' || out[i] == '-') ++i;
    if (i >= n) return false;
    bool any = false;
    while (i < n && isdigit((unsigned char)out[i])) { any = true; ++i; }
    if (i < n && out[i] == '.') {
        ++i;
        while (i < n && isdigit((unsigned char)out[i])) { any = true; ++i; }
    }
    if (!any) return false;
    if (i < n && (out[i] == 'e' || out[i] == 'E')) {
        ++i;
        if (i < n && (out[i] == '+' || out[i] == '-')) ++i;
        bool ed = false;
        while (i < n && isdigit((unsigned char)out[i])) { ed = true; ++i; }
        if (!ed) return false;
    }
    return i == n;
}

struct Sq {
    double x, y, a;
    std::string xs, ys, as;
    double cx[4], cy[4];
    double box[4];  // min_x, min_y, max_x, max_y, padded by 1e-7
};

static void float_corners(Sq& q) {
    double c = std::cos(q.a), s = std::sin(q.a);
    double ux = 0.5 * c - 0.5 * s, uy = 0.5 * s + 0.5 * c;
    double vx = -0.5 * c - 0.5 * s, vy = -0.5 * s + 0.5 * c;
    q.cx[0] = q.x + ux; q.cy[0] = q.y + uy;
    q.cx[1] = q.x + vx; q.cy[1] = q.y + vy;
    q.cx[2] = q.x - ux; q.cy[2] = q.y - uy;
    q.cx[3] = q.x - vx; q.cy[3] = q.y - vy;
    double x0 = q.cx[0], x1 = q.cx[0], y0 = q.cy[0], y1 = q.cy[0];
    for (int k = 1; k < 4; ++k) {
        x0 = std::min(x0, q.cx[k]); x1 = std::max(x1, q.cx[k]);
        y0 = std::min(y0, q.cy[k]); y1 = std::max(y1, q.cy[k]);
    }
    q.box[0] = x0 - 1e-7; q.box[1] = y0 - 1e-7; q.box[2] = x1 + 1e-7; q.box[3] = y1 + 1e-7;
}

// 1 separated, -1 overlapping, 0 undecided (threshold 1e-8).
static int float_sat(const Sq& p, const Sq& q) {
    double c1 = std::cos(p.a), s1 = std::sin(p.a), c2 = std::cos(q.a), s2 = std::sin(q.a);
    double ax[4][2] = {{c1, s1}, {-s1, c1}, {c2, s2}, {-s2, c2}};
    double worst = 1e300;
    for (auto& u : ax) {
        double lo1 = 1e300, hi1 = -1e300, lo2 = 1e300, hi2 = -1e300;
        for (int k = 0; k < 4; ++k) {
            double a = u[0] * p.cx[k] + u[1] * p.cy[k];
            double b = u[0] * q.cx[k] + u[1] * q.cy[k];
            if (a < lo1) lo1 = a;
            if (a > hi1) hi1 = a;
            if (b < lo2) lo2 = b;
            if (b > hi2) hi2 = b;
        }
        double ov = std::min(hi1, hi2) - std::max(lo1, lo2);
        if (ov < -1e-8) return 1;
        worst = std::min(worst, ov);
    }
    return worst > 1e-8 ? -1 : 0;
}

template <int F>
struct IvSq {
    bool ready = false, flat = false;
    Iv<F> c, s, x0, x1, y0, y1;
    Iv<F> px[4], py[4];
};

template <int F>
static int iv_sat(const IvSq<F>& p, const IvSq<F>& q) {
    Fx<F> z;
    auto lo_min = [](const Fx<F>& a, const Fx<F>& b) { return cmp(a, b) < 0 ? a : b; };
    auto hi_max = [](const Fx<F>& a, const Fx<F>& b) { return cmp(a, b) > 0 ? a : b; };
    if (p.flat && q.flat) {
        Iv<F> ox = isub(Iv<F>{lo_min(p.x1.lo, q.x1.lo), lo_min(p.x1.hi, q.x1.hi)},
                        Iv<F>{hi_max(p.x0.lo, q.x0.lo), hi_max(p.x0.hi, q.x0.hi)});
        if (cmp(ox.hi, z) <= 0) return 1;
        Iv<F> oy = isub(Iv<F>{lo_min(p.y1.lo, q.y1.lo), lo_min(p.y1.hi, q.y1.hi)},
                        Iv<F>{hi_max(p.y0.lo, q.y0.lo), hi_max(p.y0.hi, q.y0.hi)});
        if (cmp(oy.hi, z) <= 0) return 1;
        if (cmp(ox.lo, z) <= 0 || cmp(oy.lo, z) <= 0) return 0;
        return -1;
    }
    Iv<F> axes[4][2] = {{p.c, p.s}, {ineg(p.s), p.c}, {q.c, q.s}, {ineg(q.s), q.c}};
    bool open = false;
    for (auto& u : axes) {
        Iv<F> mn1{}, mx1{}, mn2{}, mx2{};
        for (int k = 0; k < 4; ++k) {
            Iv<F> a = iadd(imul(u[0], p.px[k]), imul(u[1], p.py[k]));
            Iv<F> b = iadd(imul(u[0], q.px[k]), imul(u[1], q.py[k]));
            if (k == 0) { mn1 = mx1 = a; mn2 = mx2 = b; continue; }
            mn1.lo = lo_min(a.lo, mn1.lo); mn1.hi = lo_min(a.hi, mn1.hi);
            mx1.lo = hi_max(a.lo, mx1.lo); mx1.hi = hi_max(a.hi, mx1.hi);
            mn2.lo = lo_min(b.lo, mn2.lo); mn2.hi = lo_min(b.hi, mn2.hi);
            mx2.lo = hi_max(b.lo, mx2.lo); mx2.hi = hi_max(b.hi, mx2.hi);
        }
        Iv<F> ov = isub(Iv<F>{lo_min(mx1.lo, mx2.lo), lo_min(mx1.hi, mx2.hi)},
                        Iv<F>{hi_max(mn1.lo, mn2.lo), hi_max(mn1.hi, mn2.hi)});
        if (cmp(ov.hi, z) <= 0) return 1;
        if (cmp(ov.lo, z) <= 0) open = true;
    }
    return open ? 0 : -1;
}

// One escalation stage at F limbs over `pairs`.  Returns -1 if a pair is
// certified overlapping, 1 if every pair is certified separated, otherwise 0
// with the still-open pairs in `left`.
template <int F>
static int stage(const std::vector<Sq>& sq, const std::vector<std::pair<int, int>>& pairs,
                 std::vector<std::pair<int, int>>& left) {
    Iv<F> ox = parse_iv<F>(sq[0].xs), oy = parse_iv<F>(sq[0].ys);
    static const Iv<F> h = parse_iv<F>("0.5");
    std::vector<IvSq<F>> cache(sq.size());
    std::unordered_map<std::string, std::pair<Iv<F>, Iv<F>>> trig;
    auto get = [&](int i) -> const IvSq<F>& {
        IvSq<F>& e = cache[(size_t)i];
        if (e.ready) return e;
        Iv<F> x = isub(parse_iv<F>(sq[(size_t)i].xs), ox), y = isub(parse_iv<F>(sq[(size_t)i].ys), oy);
        auto it = trig.find(sq[(size_t)i].as);
        if (it != trig.end()) { e.c = it->second.first; e.s = it->second.second; }
        else {
            sincos_iv(parse_iv<F>(sq[(size_t)i].as), e.s, e.c);
            trig.emplace(sq[(size_t)i].as, std::make_pair(e.c, e.s));
        }
        e.flat = e.s.lo.zero() && e.s.hi.zero();
        if (e.flat) {
            e.x0 = isub(x, h); e.x1 = iadd(x, h);
            e.y0 = isub(y, h); e.y1 = iadd(y, h);
        }
        Iv<F> hc = imul(h, e.c), hs = imul(h, e.s), nh = ineg(h);
        Iv<F> ux = isub(hc, hs), uy = iadd(hs, hc);
        Iv<F> vx = isub(imul(nh, e.c), hs), vy = iadd(imul(nh, e.s), hc);
        e.px[0] = iadd(x, ux); e.py[0] = iadd(y, uy);
        e.px[1] = iadd(x, vx); e.py[1] = iadd(y, vy);
        e.px[2] = isub(x, ux); e.py[2] = isub(y, uy);
        e.px[3] = isub(x, vx); e.py[3] = isub(y, vy);
        e.ready = true;
        return e;
    };
    left.clear();
    for (auto& pr : pairs) {
        const IvSq<F>& a = get(pr.first);
        const IvSq<F>& b = get(pr.second);
        int r = iv_sat(a, b);
        if (r < 0) return -1;
        if (r == 0) left.push_back(pr);
    }
    return left.empty() ? 1 : 0;
}

template <int F>
static std::string fifty(const Fx<F>& v) {
    uint64_t low = v.d[6] % 10000ULL, top = v.d[6] / 10000ULL;
    bool tail = false;
    for (int i = 7; i <= F; ++i) tail |= v.d[i] != 0;
    bool up = low > 5000ULL || (low == 5000ULL && (tail || (top & 1ULL)));
    uint64_t o[7] = {v.d[0], v.d[1], v.d[2], v.d[3], v.d[4], v.d[5], top};
    if (up && ++o[6] >= 100000ULL) {
        o[6] -= 100000ULL;
        int i = 5;
        for (; i >= 1; --i) {
            if (++o[i] < B9) break;
            o[i] -= B9;
        }
        if (i < 1) o[0] += 1;
    }
    bool allz = true;
    for (uint64_t w : o) allz &= w == 0;
    char buf[128];
    std::snprintf(buf, sizeof buf, "%s%llu.%09llu%09llu%09llu%09llu%09llu%05llu",
                  (v.neg && !allz) ? "-" : "", (unsigned long long)o[0], (unsigned long long)o[1],
                  (unsigned long long)o[2], (unsigned long long)o[3], (unsigned long long)o[4],
                  (unsigned long long)o[5], (unsigned long long)o[6]);
    return buf;
}

struct Verdict {
    bool ok = false;
    double score = 0;
    std::string L, reason;
};

static double grid_score(int n) { return std::ceil(std::sqrt((double)n)) / std::sqrt((double)n) - 1.0; }

static Verdict evaluate(int n, int rows, const int* sid, const char* const* xs, const char* const* ys,
                        const char* const* as) {
    Verdict v;
    v.score = grid_score(n);
    std::string N = std::to_string(n);
    if (rows != n) {
        v.reason = "n=" + N + ": expected " + N + " rows, got " + std::to_string(rows);
        return v;
    }
    std::vector<int> row_of((size_t)n, -1);
    for (int r = 0; r < rows; ++r) {
        if (sid[r] < 0 || sid[r] >= n || row_of[(size_t)sid[r]] >= 0) {
            v.reason = "n=" + N + ": square_ids should be 0.." + std::to_string(n - 1);
            return v;
        }
        row_of[(size_t)sid[r]] = r;
    }
    std::vector<Sq> sq((size_t)n);
    for (int i = 0; i < n; ++i) {
        int r = row_of[(size_t)i];
        std::string a, b, c, head = "n=" + N + ", square " + std::to_string(i) + ": ";
        if (!literal_ok(xs[r], a) || !literal_ok(ys[r], b) || !literal_ok(as[r], c)) {
            v.reason = head + "cannot parse coordinates";
            return v;
        }
        double xf = std::strtod(a.c_str(), nullptr), yf = std::strtod(b.c_str(), nullptr),
               af = std::strtod(c.c_str(), nullptr);
        if (!std::isfinite(xf) || !std::isfinite(yf) || !std::isfinite(af)) {
            v.reason = head + "value out of range for a double";
            return v;
        }
        if (std::fabs(xf) > 1e4 || std::fabs(yf) > 1e4) {
            v.reason = head + "coordinate out of bounds";
            return v;
        }
        if (std::fabs(af) > 100.0) {
            v.reason = head + "angle out of bounds";
            return v;
        }
        sq[(size_t)i].xs = a;
        sq[(size_t)i].ys = b;
        sq[(size_t)i].as = c;
    }

    using F9 = Fx<9>;
    static const F9 two_pi = parse<9>(kTwoPi, 0), half = parse<9>("0.5", 0);
    F9 x0 = parse<9>(sq[0].xs, 0), y0 = parse<9>(sq[0].ys, 0);
    std::unordered_map<std::string, std::pair<F9, F9>> trig;
    F9 bx0, bx1, by0, by1;
    for (int i = 0; i < n; ++i) {
        Sq& q = sq[(size_t)i];
        F9 dx = sub(parse<9>(q.xs, 0), x0), dy = sub(parse<9>(q.ys, 0), y0), ang = parse<9>(q.as, 0);
        long long turns = (long long)std::floor(ang.approx() / 6.283185307179586476925);
        F9 red = sub(ang, mul(F9::of(turns), two_pi, 0));
        if (red.neg && !red.zero()) red = add(red, two_pi);
        if (cmp(red, two_pi) >= 0) red = sub(red, two_pi);
        q.x = dx.approx();
        q.y = dy.approx();
        q.a = red.approx();
        float_corners(q);
        F9 sn, cs;
        if (q.as == "0" || q.as == "0.0" || ang.zero()) {
            cs = F9::of(1);
        } else {
            auto it = trig.find(q.as);
            if (it != trig.end()) { cs = it->second.first; sn = it->second.second; }
            else {
                sincos_point(ang, sn, cs);
                trig.emplace(q.as, std::make_pair(cs, sn));
            }
        }
        F9 hc = mul(half, cs, 0), hs = mul(half, sn, 0);
        F9 ux = sub(hc, hs), uy = add(hs, hc), vx = sub(F9(), add(hc, hs)), vy = sub(hc, hs);
        F9 px[4] = {add(dx, ux), add(dx, vx), sub(dx, ux), sub(dx, vx)};
        F9 py[4] = {add(dy, uy), add(dy, vy), sub(dy, uy), sub(dy, vy)};
        for (int k = 0; k < 4; ++k) {
            if (i == 0 && k == 0) { bx0 = bx1 = px[0]; by0 = by1 = py[0]; continue; }
            if (cmp(px[k], bx0) < 0) bx0 = px[k];
            if (cmp(px[k], bx1) > 0) bx1 = px[k];
            if (cmp(py[k], by0) < 0) by0 = py[k];
            if (cmp(py[k], by1) > 0) by1 = py[k];
        }
    }
    F9 wx = sub(bx1, bx0), wy = sub(by1, by0);
    F9 side = cmp(wx, wy) >= 0 ? wx : wy;

    std::vector<int> order((size_t)n);
    for (int i = 0; i < n; ++i) order[(size_t)i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return sq[(size_t)a].box[0] < sq[(size_t)b].box[0]; });
    std::vector<std::pair<int, int>> open;
    for (int u = 0; u < n; ++u) {
        const Sq& A = sq[(size_t)order[(size_t)u]];
        for (int w = u + 1; w < n; ++w) {
            const Sq& Bq = sq[(size_t)order[(size_t)w]];
            if (Bq.box[0] > A.box[2]) break;
            if (A.box[2] < Bq.box[0] || Bq.box[2] < A.box[0] || A.box[3] < Bq.box[1] || Bq.box[3] < A.box[1])
                continue;
            int i = std::min(order[(size_t)u], order[(size_t)w]), j = std::max(order[(size_t)u], order[(size_t)w]);
            int r = float_sat(sq[(size_t)i], sq[(size_t)j]);
            if (r < 0) {
                v.reason = "infeasible: Squares " + std::to_string(i) + " and " + std::to_string(j) +
                           " overlap (float check)";
                return v;
            }
            if (r == 0) open.emplace_back(i, j);
        }
    }
    if (!open.empty()) {
        std::vector<std::pair<int, int>> l1, l2, l3;
        int r = stage<7>(sq, open, l1);
        if (r == 0) r = stage<15>(sq, l1, l2);
        if (r == 0) {
            r = stage<58>(sq, l2, l3);
            if (r == 0) {
                v.reason = "infeasible: Overlap undecidable at max precision";
                return v;
            }
        }
        if (r < 0) {
            v.reason = "infeasible: Squares overlap (certified)";
            return v;
        }
    }
    double sf = side.approx(), lb = std::sqrt((double)n);
    if (sf < lb - 1e-7) {
        v.reason = "infeasible: L is below area lower bound";
        return v;
    }
    v.ok = true;
    v.reason = "ok";
    v.L = fifty(side);
    v.score = std::max(0.0, sf / lb - 1.0);
    return v;
}

static void put(char* dst, int cap, const std::string& s) {
    if (!dst || cap <= 0) return;
    size_t k = std::min((size_t)cap - 1, s.size());
    std::memcpy(dst, s.data(), k);
    dst[k] = 0;
}

}  // namespace orc

extern "C" {

// One packing.  Returns 1 when accepted (L_out holds the 50-decimal side), 0
// when rejected (reason_out holds the reason).
int sqo_certify(int n, int rows, const int* sid, const char* const* xs, const char* const* ys,
                const char* const* as, char* L_out, int L_cap, char* reason_out, int reason_cap,
                double* score) {
    orc::Verdict v = orc::evaluate(n, rows, sid, xs, ys, as);
    orc::put(L_out, L_cap, v.ok ? v.L : std::string());
    orc::put(reason_out, reason_cap, v.reason);
    if (score) *score = v.score;
    return v.ok ? 1 : 0;
}

// Pandas transport emulation: shortest of %.15g/%.16g/%.17g that reads back
// to the same double, with ".0" appended to a bare integer.
void sqo_roundtrip(const char* s, char* out, int cap) {
    double v = std::strtod(s, nullptr);
    char buf[64];
    for (int p = 15; p <= 17; ++p) {
        std::snprintf(buf, sizeof buf, "%.*g", p, v);
        if (std::strtod(buf, nullptr) == v) break;
    }
    std::string r(buf);
    if (r.find_first_of(".eE") == std::string::npos) r += ".0";
    orc::put(out, cap, r);
}

}  // extern "C"

#include <atomic>
#include <thread>

// Batch form of sqo_certify, threaded over packings (the layout of
// ref_evaluate_batch in ref_certifier.cpp).
// The same with each packing's 50-decimal side and reason written to
// L_out + 80 p and reason_out + 112 p (either may be NULL).
extern "C" int sqo_certify_batch_text(int count, const int* n_of, const long long* row_start, const int* sid,
                                      const char* text, const long long* lit_off, int threads, int* ok_out,
                                      double* score_out, char* L_out, char* reason_out);

extern "C" int sqo_certify_batch(int count, const int* n_of, const long long* row_start, const int* sid,
                                 const char* text, const long long* lit_off, int threads, int* ok_out,
                                 double* score_out) {
    return sqo_certify_batch_text(count, n_of, row_start, sid, text, lit_off, threads, ok_out, score_out, nullptr,
                                  nullptr);
}

static void put_text(char* dst, size_t cap, const std::string& s) {
    const size_t k = std::min(cap - 1, s.size());
    std::memcpy(dst, s.data(), k);
    dst[k] = 0;
}

extern "C" int sqo_certify_batch_text(int count, const int* n_of, const long long* row_start, const int* sid,
                                      const char* text, const long long* lit_off, int threads, int* ok_out,
                                      double* score_out, char* L_out, char* reason_out) {
    std::atomic<int> next{0};
    auto work = [&]() {
        for (int p = next.fetch_add(1); p < count; p = next.fetch_add(1)) {
            const long long r0 = row_start[p], rows = row_start[p + 1] - r0;
            std::vector<std::string> xs, ys, as;
            std::vector<int> ids;
            for (long long r = r0; r < r0 + rows; ++r) {
                ids.push_back(sid ? sid[r] : (int)(r - r0));
                xs.emplace_back(text + lit_off[3 * r], (size_t)(lit_off[3 * r + 1] - lit_off[3 * r]));
                ys.emplace_back(text + lit_off[3 * r + 1], (size_t)(lit_off[3 * r + 2] - lit_off[3 * r + 1]));
                as.emplace_back(text + lit_off[3 * r + 2], (size_t)(lit_off[3 * r + 3] - lit_off[3 * r + 2]));
            }
            std::vector<const char*> px, py, pa;
            for (long long k = 0; k < rows; ++k) {
                px.push_back(xs[(size_t)k].c_str());
                py.push_back(ys[(size_t)k].c_str());
                pa.push_back(as[(size_t)k].c_str());
            }
            orc::Verdict v = orc::evaluate(n_of[p], (int)rows, ids.data(), px.data(), py.data(), pa.data());
            ok_out[p] = v.ok ? 1 : 0;
            if (score_out) score_out[p] = v.score;
            if (L_out) put_text(L_out + 80 * (size_t)p, 80, v.ok ? v.L : std::string());
            if (reason_out) put_text(reason_out + 112 * (size_t)p, 112, v.reason);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
    return threads;
}
