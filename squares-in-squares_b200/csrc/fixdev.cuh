// Signed fixed-point numbers in base 1e9 (one integer limb, F fraction limbs)
// and closed intervals of them -- host and device.
//
// The certifier's verdicts and its 50-decimal side must equal the reference
// certifier's bit for bit, so every operation below reproduces the reference
// arithmetic exactly (cuda/certifier.cpp:32-503): truncating decimal parse,
// multiplication rounded half-up on the first dropped limb or directed
// (toward -inf / +inf) on any non-zero dropped limb, division by a small
// integer rounded half-up, a zero that is never negative, the 1-ulp widening
// of non-dyadic literals and of Taylor-series hulls, and the quadrant
// reduction of sin/cos from a double estimate.
//
// Representation for the GPU: 32-bit limbs (< 1e9).  Products of two limbs
// are < 1e18, so a column of up to 16 products plus its carry fits a u64;
// the 58-limb stage splits its columns.  The integer limb never exceeds a few
// thousand here (coordinates are bounded by 1e4 before any arithmetic).
#pragma once
#include <cstdint>
#ifdef __CUDACC__
#define FX_HD __host__ __device__ __forceinline__
// Multi-limb routines stay out of line: inlined and unrolled at 58 limbs they
// exhaust the register file and the compiler's patience.
#define FX_HEAVY __host__ __device__ __noinline__
#else
#define FX_HD inline
#define FX_HEAVY inline
#endif

namespace sqs {
namespace fx {

constexpr uint32_t B9 = 1000000000u;
// Widest fraction whose comparison and addition a caller may ask to have
// inlined (the 7-limb interval SAT test and the 9-limb side measurement:
// values stay in registers).
constexpr int kInlineLimbs = 9;

template <int F>
struct Fix {
    uint32_t d[F + 1];  // d[0] integer limb, d[1..F] fraction limbs (most significant first)
    uint32_t neg;       // 1 when negative; zero is stored non-negative
};

template <int F>
FX_HD void set_zero(Fix<F>& a) {
    for (int i = 0; i <= F; ++i) a.d[i] = 0;
    a.neg = 0;
}

template <int F>
FX_HD Fix<F> of_int(long long v) {
    Fix<F> r;
    set_zero(r);
    if (v < 0) { r.neg = 1; v = -v; }
    r.d[0] = (uint32_t)v;
    return r;
}

template <int F>
FX_HD bool is_zero(const Fix<F>& a) {
    uint32_t o = 0;
    for (int i = 0; i <= F; ++i) o |= a.d[i];
    return o == 0;
}

template <int F>
FX_HD void fix_zero(Fix<F>& a) {
    if (is_zero(a)) a.neg = 0;
}

// The reference's to_double: integer limb plus at most four fraction limbs,
// each scaled by a running product of 1e-9 (same operation order).
template <int F>
FX_HD double approx(const Fix<F>& a) {
    double v = (double)a.d[0], sc = 1.0;
    constexpr int K = F < 4 ? F : 4;
    for (int i = 1; i <= K; ++i) {
        sc *= 1e-9;
        v += (double)a.d[i] * sc;
    }
    return a.neg ? -v : v;
}

template <int F, bool IN>
FX_HD int mag_cmp_body(const Fix<F>& a, const Fix<F>& b) {
    for (int i = 0; i <= F; ++i)
        if (a.d[i] != b.d[i]) return a.d[i] < b.d[i] ? -1 : 1;
    return 0;
}
template <int F>
FX_HEAVY int mag_cmp_out(const Fix<F>& a, const Fix<F>& b) { return mag_cmp_body<F, false>(a, b); }
// IN: inline at up to kInlineLimbs limbs (for the interval SAT test);
// otherwise the out-of-line routine
template <int F, bool IN = false>
FX_HD int mag_cmp(const Fix<F>& a, const Fix<F>& b) {
    if constexpr (IN && F <= kInlineLimbs) return mag_cmp_body<F, true>(a, b);
    else return mag_cmp_out<F>(a, b);
}

template <int F, bool IN>
FX_HD int cmp_body(const Fix<F>& a, const Fix<F>& b) {
    const bool za = is_zero(a), zb = is_zero(b);
    if (za && zb) return 0;
    if (a.neg != b.neg) return a.neg ? -1 : 1;
    const int c = mag_cmp<F, IN>(a, b);
    return a.neg ? -c : c;
}
template <int F>
FX_HEAVY int cmp_out(const Fix<F>& a, const Fix<F>& b) { return cmp_body<F, false>(a, b); }
// IN: inline at up to kInlineLimbs limbs (for the interval SAT test);
// otherwise the out-of-line routine
template <int F, bool IN = false>
FX_HD int cmp(const Fix<F>& a, const Fix<F>& b) {
    if constexpr (IN && F <= kInlineLimbs) return cmp_body<F, true>(a, b);
    else return cmp_out<F>(a, b);
}

template <int F, bool IN>
FX_HD Fix<F> mag_add_body(const Fix<F>& a, const Fix<F>& b, uint32_t neg) {
    Fix<F> r;
    uint32_t c = 0;
    for (int i = F; i >= 1; --i) {
        uint32_t s = a.d[i] + b.d[i] + c;  // < 2e9 + 1 < 2^32
        c = s >= B9;
        r.d[i] = c ? s - B9 : s;
    }
    r.d[0] = a.d[0] + b.d[0] + c;
    r.neg = neg;
    fix_zero(r);
    return r;
}
template <int F>
FX_HEAVY Fix<F> mag_add_out(const Fix<F>& a, const Fix<F>& b, uint32_t neg) { return mag_add_body<F, false>(a, b, neg); }
// IN: inline at up to kInlineLimbs limbs (for the interval SAT test);
// otherwise the out-of-line routine
template <int F, bool IN = false>
FX_HD Fix<F> mag_add(const Fix<F>& a, const Fix<F>& b, uint32_t neg) {
    if constexpr (IN && F <= kInlineLimbs) return mag_add_body<F, true>(a, b, neg);
    else return mag_add_out<F>(a, b, neg);
}

template <int F, bool IN>
FX_HD Fix<F> mag_sub_body(const Fix<F>& a, const Fix<F>& b, uint32_t neg) {  // |a| >= |b|
    Fix<F> r;
    uint32_t br = 0;
    for (int i = F; i >= 1; --i) {
        const uint32_t sub = b.d[i] + br;
        br = a.d[i] < sub;
        r.d[i] = br ? a.d[i] + B9 - sub : a.d[i] - sub;
    }
    r.d[0] = a.d[0] - b.d[0] - br;
    r.neg = neg;
    fix_zero(r);
    return r;
}
template <int F>
FX_HEAVY Fix<F> mag_sub_out(const Fix<F>& a, const Fix<F>& b, uint32_t neg) { return mag_sub_body<F, false>(a, b, neg); }
// IN: inline at up to kInlineLimbs limbs (for the interval SAT test);
// otherwise the out-of-line routine
template <int F, bool IN = false>
FX_HD Fix<F> mag_sub(const Fix<F>& a, const Fix<F>& b, uint32_t neg) {
    if constexpr (IN && F <= kInlineLimbs) return mag_sub_body<F, true>(a, b, neg);
    else return mag_sub_out<F>(a, b, neg);
}

template <int F, bool IN>
FX_HD Fix<F> add_body(const Fix<F>& a, const Fix<F>& b) {
    if (a.neg == b.neg) return mag_add<F, IN>(a, b, a.neg);
    const int c = mag_cmp<F, IN>(a, b);
    if (c == 0) {
        Fix<F> z;
        set_zero(z);
        return z;
    }
    return c > 0 ? mag_sub<F, IN>(a, b, a.neg) : mag_sub<F, IN>(b, a, b.neg);
}
template <int F>
FX_HEAVY Fix<F> add_out(const Fix<F>& a, const Fix<F>& b) { return add_body<F, false>(a, b); }
// IN: inline at up to kInlineLimbs limbs (for the interval SAT test);
// otherwise the out-of-line routine
template <int F, bool IN = false>
FX_HD Fix<F> add(const Fix<F>& a, const Fix<F>& b) {
    if constexpr (IN && F <= kInlineLimbs) return add_body<F, true>(a, b);
    else return add_out<F>(a, b);
}

template <int F>
FX_HD Fix<F> neg(Fix<F> a) {
    a.neg ^= 1u;
    fix_zero(a);
    return a;
}

template <int F, bool IN = false>
FX_HD Fix<F> sub(const Fix<F>& a, const Fix<F>& b) { return add<F, IN>(a, neg(b)); }

template <int F>
FX_HD void bump(Fix<F>& a) {  // |a| += 1 unit of the last limb
    for (int i = F; i >= 1; --i) {
        if (++a.d[i] < B9) return;
        a.d[i] = 0;
    }
    a.d[0] += 1;
}

// Exact product limbs p[0..2F] (p[0] keeps the integer part modulo 1e9, as the
// reference's row-wise carry does), column by column.
template <int F>
FX_HEAVY void mul_limbs(const Fix<F>& a, const Fix<F>& b, uint32_t* p) {
    uint64_t carry = 0;
    for (int k = 2 * F; k >= 0; --k) {
        const int lo = k - F > 0 ? k - F : 0, hi = k < F ? k : F;
        uint64_t s = carry, over = 0;
        int cnt = 0;
        for (int i = lo; i <= hi; ++i) {
            s += (uint64_t)a.d[i] * (uint64_t)b.d[k - i];
            if (++cnt == 16) {  // keep the column sum below 2^64
                over += s / B9;
                s %= B9;
                cnt = 0;
            }
        }
        p[k] = (uint32_t)(s % B9);
        carry = over + s / B9;
    }
}

// rnd: 0 = half-up on the first dropped limb; -1 / +1 = directed.
template <int F>
FX_HEAVY Fix<F> mul(const Fix<F>& a, const Fix<F>& b, int rnd) {
    Fix<F> r;
    if (is_zero(a) || is_zero(b)) {
        set_zero(r);
        return r;
    }
    uint32_t p[2 * F + 1];
    mul_limbs(a, b, p);
    for (int i = 0; i <= F; ++i) r.d[i] = p[i];
    r.neg = a.neg ^ b.neg;
    if (rnd == 0) {
        if (p[F + 1] >= B9 / 2) bump(r);
    } else {
        uint32_t tail = 0;
        for (int i = F + 1; i <= 2 * F; ++i) tail |= p[i];
        if (tail && ((rnd > 0) == (r.neg == 0))) bump(r);
    }
    fix_zero(r);
    return r;
}

FX_HD uint64_t mulhi64(uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
    return __umul64hi(a, b);
#else
    return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

// Division of t < 2^64 by a divisor d fixed across many calls, through the
// reciprocal m = floor((2^64 - 1) / d) computed once: q = floor(t m / 2^64)
// never exceeds t / d and falls short of it by less than 3, so at most two
// corrections make the quotient and remainder exact.  (Division by an
// invariant integer through multiplication, after Granlund and Montgomery.)
struct Recip {
    uint64_t m;
    uint64_t d;
};
FX_HD Recip recip(uint32_t d) { return Recip{~0ull / d, d}; }
FX_HD uint64_t div_rem(uint64_t t, const Recip& R, uint64_t& rem) {
    uint64_t q = mulhi64(t, R.m);
    uint64_t r = t - q * R.d;
    while (r >= R.d) {
        ++q;
        r -= R.d;
    }
    rem = r;
    return q;
}

template <int F>
FX_HEAVY Fix<F> div_small(const Fix<F>& a, uint32_t den) {  // half-up on the remainder
    Fix<F> r;
    const Recip R = recip(den);
    uint64_t rem = 0;
    for (int i = 0; i <= F; ++i) {
        const uint64_t t = rem * B9 + a.d[i];  // rem < den < 2^32: t < 2^64
        r.d[i] = (uint32_t)div_rem(t, R, rem);
    }
    r.neg = a.neg;
    if (rem * 2 >= den) bump(r);
    fix_zero(r);
    return r;
}

template <int F>
struct Iv {
    Fix<F> lo, hi;
};

template <int F, bool IN = false>
FX_HD Iv<F> iadd(const Iv<F>& a, const Iv<F>& b) { return {add<F, IN>(a.lo, b.lo), add<F, IN>(a.hi, b.hi)}; }
template <int F, bool IN = false>
FX_HD Iv<F> isub(const Iv<F>& a, const Iv<F>& b) { return {sub<F, IN>(a.lo, b.hi), sub<F, IN>(a.hi, b.lo)}; }
template <int F>
FX_HD Iv<F> ineg(const Iv<F>& a) { return {neg(a.hi), neg(a.lo)}; }
// 1: the interval is >= 0; -1: it is <= 0; 0: it straddles zero.
template <int F>
FX_HD int sign_class(const Iv<F>& a) {
    if (!a.lo.neg) return 1;
    if (a.hi.neg || is_zero(a.hi)) return -1;
    return 0;
}

// Interval product: the lower bound is the smallest of the four endpoint
// products rounded toward -inf, the upper the largest rounded toward +inf
// (the reference's imul).  Directed rounding is monotone, so the smallest
// rounded product is the rounded smallest product: the sign cases below pick
// the endpoints that give the exact extremes and round only those, with the
// same bounds as rounding all four products both ways.
template <int F>
FX_HEAVY Iv<F> imul(const Iv<F>& a, const Iv<F>& b) {
    const int sa = sign_class(a), sb = sign_class(b);
    const Fix<F>*lx, *ly, *hx, *hy;  // endpoints of the extreme products
    if (sa == 0 && sb == 0) {
        const Fix<F> d1 = mul(a.lo, b.hi, -1), d2 = mul(a.hi, b.lo, -1);
        const Fix<F> u1 = mul(a.lo, b.lo, +1), u2 = mul(a.hi, b.hi, +1);
        return Iv<F>{cmp(d1, d2) <= 0 ? d1 : d2, cmp(u1, u2) >= 0 ? u1 : u2};
    }
    if (sa > 0) {
        if (sb > 0) { lx = &a.lo; ly = &b.lo; hx = &a.hi; hy = &b.hi; }
        else if (sb < 0) { lx = &a.hi; ly = &b.lo; hx = &a.lo; hy = &b.hi; }
        else { lx = &a.hi; ly = &b.lo; hx = &a.hi; hy = &b.hi; }
    } else if (sa < 0) {
        if (sb > 0) { lx = &a.lo; ly = &b.hi; hx = &a.hi; hy = &b.lo; }
        else if (sb < 0) { lx = &a.hi; ly = &b.hi; hx = &a.lo; hy = &b.lo; }
        else { lx = &a.lo; ly = &b.hi; hx = &a.lo; hy = &b.lo; }
    } else {
        if (sb > 0) { lx = &a.lo; ly = &b.hi; hx = &a.hi; hy = &b.hi; }
        else { lx = &a.hi; ly = &b.lo; hx = &a.lo; hy = &b.lo; }
    }
    return Iv<F>{mul(*lx, *ly, -1), mul(*hx, *hy, +1)};
}

// ------------------------------------------------------------ decimal literals
// A validated literal after whitespace stripping: sign, mantissa digits (the
// dot skipped) and the position of the decimal point after the exponent.
struct Lit {
    uint32_t off;    // text offset of the first mantissa character (after the sign)
    int32_t point;   // number of digits before the decimal point (may be <= 0 or > ndig)
    uint16_t ndig;   // mantissa digit count
    int16_t dot;     // index (in digits) where the '.' sits, or -1
    uint8_t neg;     // leading '-'
    uint8_t dyadic;  // finite binary expansion within 25 decimal places
    uint8_t zero_str;// the stripped literal is exactly "0" or "0.0"
    uint8_t pad;
};

FX_HD int lit_digit(const char* text, const Lit& L, long long k) {
    if (k < 0 || k >= L.ndig) return 0;
    const long long c = (long long)L.off + k + ((L.dot >= 0 && k >= L.dot) ? 1 : 0);
    return text[c] - '0';
}

// parse_decimal_fix: truncation (rnd 0) or directed rounding of the magnitude.
template <int F>
FX_HEAVY Fix<F> parse(const char* text, const Lit& L, int rnd) {
    Fix<F> r;
    uint32_t iv = 0;
    for (long long k = 0; k < L.point; ++k) iv = iv * 10u + (uint32_t)lit_digit(text, L, k);
    r.d[0] = iv;
    for (int l = 1; l <= F; ++l) {
        uint32_t v = 0;
        const long long base = (long long)L.point + (long long)(l - 1) * 9;
        for (int k = 0; k < 9; ++k) v = v * 10u + (uint32_t)lit_digit(text, L, base + k);
        r.d[l] = v;
    }
    r.neg = L.neg;
    bool tail = false;
    long long start = (long long)L.point + 9LL * F;
    if (start < 0) start = 0;
    for (long long pos = start; pos < L.ndig && !tail; ++pos) tail = lit_digit(text, L, pos) != 0;
    if (tail && rnd != 0 && ((rnd > 0) == (L.neg == 0))) bump(r);
    fix_zero(r);
    return r;
}

template <int F>
FX_HEAVY Iv<F> parse_iv(const char* text, const Lit& L) {
    Iv<F> r{parse<F>(text, L, -1), parse<F>(text, L, +1)};
    if (!L.dyadic) {
        Fix<F> u;
        set_zero(u);
        u.d[F] = 1;
        r.lo = sub(r.lo, u);
        r.hi = add(r.hi, u);
    }
    return r;
}

// ------------------------------------------------------------ sin / cos
template <int F>
FX_HEAVY void taylor(const Fix<F>& x, Fix<F>& sn, Fix<F>& cs, int terms) {
    const Fix<F> x2 = mul(x, x, 0);
    Fix<F> ct = of_int<F>(1), st = x;
    cs = of_int<F>(1);
    sn = x;
    for (int m = 1; m <= terms; ++m) {
        ct = div_small(mul(ct, x2, 0), (uint32_t)((2 * m - 1) * (2 * m)));
        ct.neg = (uint32_t)(m & 1);
        fix_zero(ct);
        cs = add(cs, ct);
        st = div_small(mul(st, x2, 0), (uint32_t)((2 * m) * (2 * m + 1)));
        st.neg = (m & 1) ? (x.neg ^ 1u) : x.neg;
        fix_zero(st);
        sn = add(sn, st);
        if (is_zero(ct) && is_zero(st)) break;
    }
}

FX_HD double round_half_away(double v) {
#ifdef __CUDA_ARCH__
    return round(v);
#else
    return __builtin_round(v);
#endif
}

// Point sin/cos (the side measurement): quadrant q from the double estimate.
template <int F>
FX_HEAVY void sincos_point(const Fix<F>& a, const Fix<F>& half_pi, Fix<F>& sn, Fix<F>& cs) {
    const long long q = (long long)round_half_away(approx(a) / 1.57079632679489661923);
    const Fix<F> r = sub(a, mul(of_int<F>(q), half_pi, 0));
    Fix<F> s0, c0;
    taylor(r, s0, c0, F <= 10 ? 32 : 115);
    switch ((int)((q % 4 + 4) % 4)) {
        case 0: sn = s0; cs = c0; break;
        case 1: sn = c0; cs = neg(s0); break;
        case 2: sn = neg(s0); cs = neg(c0); break;
        default: sn = neg(c0); cs = s0; break;
    }
}

// Interval sin/cos: Taylor at both reduced endpoints, hull widened one ulp,
// cos raised to 1 when the reduced interval touches 0.
template <int F>
FX_HEAVY void sincos_iv(const Iv<F>& a, const Iv<F>& half_pi, Iv<F>& sn, Iv<F>& cs) {
    if (is_zero(a.lo) && is_zero(a.hi)) {
        set_zero(sn.lo);
        set_zero(sn.hi);
        cs.lo = of_int<F>(1);
        cs.hi = of_int<F>(1);
        return;
    }
    const double mid = 0.5 * (approx(a.lo) + approx(a.hi));
    const long long q = (long long)round_half_away(mid / 1.57079632679489661923);
    const Fix<F> qf = of_int<F>(q);
    const Iv<F> r = isub(a, imul(Iv<F>{qf, qf}, half_pi));
    const int terms = F <= 8 ? 28 : (F <= 15 ? 45 : 145);
    Fix<F> sl, cl, sh, ch;
    taylor(r.lo, sl, cl, terms);
    if (cmp(r.lo, r.hi) == 0) {
        sh = sl;
        ch = cl;
    } else {
        taylor(r.hi, sh, ch, terms);
    }
    Fix<F> e;
    set_zero(e);
    e.d[F] = 1;
    const Fix<F> one = of_int<F>(1);
    Iv<F> s0{cmp(sl, sh) < 0 ? sl : sh, cmp(sl, sh) > 0 ? sl : sh};
    Iv<F> c0{cmp(cl, ch) < 0 ? cl : ch, cmp(cl, ch) > 0 ? cl : ch};
    s0.lo = sub(s0.lo, e);
    s0.hi = add(s0.hi, e);
    c0.lo = sub(c0.lo, e);
    c0.hi = add(c0.hi, e);
    const bool through0 = (r.lo.neg && !r.hi.neg) || is_zero(r.lo) || is_zero(r.hi);
    if (through0 && cmp(c0.hi, one) < 0) c0.hi = one;
    switch ((int)((q % 4 + 4) % 4)) {
        case 0: sn = s0; cs = c0; break;
        case 1: sn = c0; cs = ineg(s0); break;
        case 2: sn = ineg(s0); cs = ineg(c0); break;
        default: sn = ineg(c0); cs = s0; break;
    }
}

}  // namespace fx
}  // namespace sqs
