// FP32 separating-axis (SAT) penetration of two unit squares, with the
// gradient for both squares from one evaluation.
//
// Model (reference seeded.cu:41-65, pair_cached): for squares p and q with
// angles a_p, a_q, centre offset (dx, dy) = q - p, the four candidate axes
// are p's (cos a_p, sin a_p), (-sin a_p, cos a_p) and q's two.  Along every
// axis both squares have the same support radius
//     r = 1/2 + 1/2 (|cos(a_q - a_p)| + |sin(a_q - a_p)|),
// so the signed gap along axis k is |v_k| - r with v_k the projection of
// the offset.  gap = max_k; the pair energy is gap^2 when gap < 0 (the
// squares overlap) and 0 otherwise, and 0 whenever |offset|^2 >= 2.000001.
//
// The reference evaluates pair(p, q) for the gradient of p and pair(q, p)
// for the gradient of q, picking the first maximal axis in its own order
// (own axes first).  Here one evaluation serves both: p's gradient uses the
// first maximum in axis order (0,1,2,3), q's in order (2,3,0,1), which is
// exactly what pair(q, p) would pick, so the per-square gradients equal the
// reference's sums over pairs even at ties (aligned squares).
#pragma once
#include <cuda_runtime.h>

namespace sqs {

constexpr float kPairCut2 = 2.000001f;  // seeded.cu:43

// sign(v) in {-1, 0, 1} with selects only (no integer -> float conversion).
__device__ __forceinline__ float sgnf(float v) { return v > 0.f ? 1.f : (v < 0.f ? -1.f : 0.f); }

struct PairGrad {
    float e;            // gap^2
    float px, py, pa;   // d e / d p
    float qx, qy, qa;   // d e / d q
};

// Evaluate an overlapping pair.  Returns false (and leaves g untouched) when
// the squares do not overlap.  cp, sp: cos/sin of p's angle; cq, sq of q's.
__device__ __forceinline__ bool sat_pair_grad(float dx, float dy, float cp, float sp, float cq,
                                              float sq, PairGrad& g) {
    // Products kept unfused so that equal angles give sd == 0 exactly.
    const float cd = __fadd_rn(__fmul_rn(cp, cq), __fmul_rn(sp, sq));
    const float sd = __fsub_rn(__fmul_rn(sp, cq), __fmul_rn(cp, sq));
    const float rad = 0.5f + 0.5f * (fabsf(cd) + fabsf(sd));
    const float v0 = dx * cp + dy * sp;
    const float v1 = dy * cp - dx * sp;
    const float v2 = dx * cq + dy * sq;
    const float v3 = dy * cq - dx * sq;
    const float z0 = fabsf(v0) - rad, z1 = fabsf(v1) - rad;
    const float z2 = fabsf(v2) - rad, z3 = fabsf(v3) - rad;
    const float gap = fmaxf(fmaxf(z0, z1), fmaxf(z2, z3));
    if (!(gap < 0.f)) return false;
    const float deriv = 0.5f * (sgnf(sd) * cd - sgnf(cd) * sd);
    const float two_gap = 2.f * gap;
    g.e = gap * gap;
    // Without a tie both squares use the same axis: one selection serves both.
    const int ties = (z0 == gap) + (z1 == gap) + (z2 == gap) + (z3 == gap);
    if (ties == 1) {
        const bool k0 = z0 == gap, k1 = z1 == gap, k2 = z2 == gap;
        const float ux = k0 ? cp : (k1 ? -sp : (k2 ? cq : -sq));
        const float uy = k0 ? sp : (k1 ? cp : (k2 ? sq : cq));
        const float v = k0 ? v0 : (k1 ? v1 : (k2 ? v2 : v3));
        const float tv = k0 ? v1 : (k1 ? -v0 : (k2 ? v3 : -v2));  // d v / d(own angle)
        const float s = sgnf(v);
        const float tp = (k0 || k1) ? s * tv : 0.f, tq = (k0 || k1) ? 0.f : s * tv;
        g.px = -two_gap * s * ux;
        g.py = -two_gap * s * uy;
        g.pa = two_gap * (tp - deriv);
        g.qx = -g.px;
        g.qy = -g.py;
        g.qa = two_gap * (tq + deriv);
        return true;
    }
    // first maximum in order 0,1,2,3 (gradient of p), as selects
    {
        const bool k0 = z0 == gap, k1 = !k0 && z1 == gap, k2 = !k0 && !k1 && z2 == gap;
        const float ux = k0 ? cp : (k1 ? -sp : (k2 ? cq : -sq));
        const float uy = k0 ? sp : (k1 ? cp : (k2 ? sq : cq));
        const float v = k0 ? v0 : (k1 ? v1 : (k2 ? v2 : v3));
        const float torque = k0 ? sgnf(v0) * v1 : (k1 ? -sgnf(v1) * v0 : 0.f);
        const float s = sgnf(v);
        g.px = -two_gap * s * ux;
        g.py = -two_gap * s * uy;
        g.pa = two_gap * (torque - deriv);
    }
    // first maximum in order 2,3,0,1 (gradient of q)
    {
        const bool k2 = z2 == gap, k3 = !k2 && z3 == gap, k0 = !k2 && !k3 && z0 == gap;
        const float ux = k2 ? cq : (k3 ? -sq : (k0 ? cp : -sp));
        const float uy = k2 ? sq : (k3 ? cq : (k0 ? sp : cp));
        const float v = k2 ? v2 : (k3 ? v3 : (k0 ? v0 : v1));
        const float torque = k2 ? sgnf(v2) * v3 : (k3 ? -sgnf(v3) * v2 : 0.f);
        const float s = sgnf(v);
        g.qx = two_gap * s * ux;
        g.qy = two_gap * s * uy;
        g.qa = two_gap * (torque + deriv);
    }
    return true;
}

// Energy only (no gradient): gap^2 or 0.  Same axis model.  Every rounding
// is spelled out so that the value is the same bit for bit when the two
// squares swap roles (offset negated, p's and q's cos/sin exchanged): the
// annealer adds a moved square's pair terms from its own side and takes the
// total from the lower index's, and the two must agree exactly.
__device__ __forceinline__ float sat_pair_energy(float dx, float dy, float cp, float sp, float cq,
                                                 float sq) {
    const float cd = __fadd_rn(__fmul_rn(cp, cq), __fmul_rn(sp, sq));
    const float sd = __fsub_rn(__fmul_rn(sp, cq), __fmul_rn(cp, sq));
    const float rad = 0.5f + 0.5f * (fabsf(cd) + fabsf(sd));
    const float z0 = fabsf(__fmaf_rn(dx, cp, __fmul_rn(dy, sp)));
    const float z1 = fabsf(__fmaf_rn(dy, cp, -__fmul_rn(dx, sp)));
    const float z2 = fabsf(__fmaf_rn(dx, cq, __fmul_rn(dy, sq)));
    const float z3 = fabsf(__fmaf_rn(dy, cq, -__fmul_rn(dx, sq)));
    const float gap = fmaxf(fmaxf(z0, z1), fmaxf(z2, z3)) - rad;
    return gap < 0.f ? gap * gap : 0.f;
}

// Wall penalty of one square in [0, L]^2 (reference seeded.cu:96-113 with the
// dr_smooth angle derivative, seeded.cu:36-38): sum over the four sides of
// max(0, violation)^2 where the square's half-extent is r = (|c| + |s|) / 2.
__device__ __forceinline__ float wall_energy_grad(float x, float y, float c, float s, float L,
                                                  float& gx, float& gy, float& ga) {
    const float r = 0.5f * (fabsf(c) + fabsf(s));
    const float sc = (fabsf(c) > 1e-6f) ? (c >= 0.f ? 1.f : -1.f) : 0.f;
    const float ss = (fabsf(s) > 1e-6f) ? (s >= 0.f ? 1.f : -1.f) : 0.f;
    const float dr = 0.5f * (-sc * s + ss * c);
    float e = 0.f;
    const float v0 = r - x, v1 = x + r - L, v2 = r - y, v3 = y + r - L;
    if (v0 > 0.f) { e += v0 * v0; gx -= 2.f * v0; ga += 2.f * v0 * dr; }
    if (v1 > 0.f) { e += v1 * v1; gx += 2.f * v1; ga += 2.f * v1 * dr; }
    if (v2 > 0.f) { e += v2 * v2; gy -= 2.f * v2; ga += 2.f * v2 * dr; }
    if (v3 > 0.f) { e += v3 * v3; gy += 2.f * v3; ga += 2.f * v3 * dr; }
    return e;
}

__device__ __forceinline__ float wall_energy(float x, float y, float c, float s, float L) {
    const float r = 0.5f * (fabsf(c) + fabsf(s));
    const float v0 = fmaxf(0.f, r - x), v1 = fmaxf(0.f, x + r - L);
    const float v2 = fmaxf(0.f, r - y), v3 = fmaxf(0.f, y + r - L);
    return v0 * v0 + v1 * v1 + v2 * v2 + v3 * v3;
}

}  // namespace sqs
