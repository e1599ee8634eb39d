// Initial states of a search's chains: the reference's structured portfolio
// (build_portfolio, seeded.cu:233-425, and the per-chain jitter of
// structured_init, seeded.cu:427-451), host code.
//
// Chain b belongs to ladder b / 8 and takes group b % 8 of it:
//   groups 0-1  the seed (ladders 0-1) or topology candidate (ladder - 2);
//   groups 2-4  topology candidate `ladder` (both modulo the candidate count);
//   groups 5-6  a cx x cy corner grid (group 6 without its far corner), up to
//               three corner anchors, the rest in two tilted rows along the
//               right and top edges of a box of side max(sqrt n + 0.05, L - 0.03);
//   group 7     four corner anchors and a rotated grid of the rest in a box of
//               side max(sqrt n + 0.05, L - 0.02)
// (groups 2-4 fall back to the group-7 layout when there is no candidate).
// A topology candidate of side L' packs corner triangles of a1, a2, b1, b2
// axis-aligned squares (bottom-left, top-right, top-left, bottom-right) and
// a band of w rows of squares at 45 degrees along the main diagonal, each row
// clipped by the container and by the b1 / b2 triangles; candidates with
// room for n to n + 4 squares and sides in [sqrt n - 0.05, L + 0.15] are
// kept, the 64 smallest.  The arithmetic is written term for term as the
// reference evaluates it, so the layouts are the reference's bit for bit
// (tested against it).  The jitter -- none for group 0, 1e-4 * 100^u for
// group 1, 0.03 otherwise, uniform in +-jitter on every coordinate and angle,
// centres kept in [0.5, L - 0.5] -- draws from this library's generator, not
// the reference's.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace sqs {
namespace port {

struct Pt {
    double x, y, a;
};

constexpr double kEps = 1e-7;

struct Topo {
    double L;
    std::vector<Pt> pts;
};

// The v-range of tilted row u in a container of side L, clipped by the b1
// (top-left) and b2 (bottom-right) triangles; valid when hi >= lo.
struct Row {
    double lo, hi;
};

static Row band_row(double u, double L, int b1, int b2, bool clip) {
    const double s2 = std::sqrt(2.0), inv_s2 = 1.0 / s2;
    Row r;
    r.lo = -std::min(u - 1.0 - kEps, s2 * L - u - 1.0 - kEps);
    r.hi = std::min(u - 1.0 - kEps, s2 * L - u - 1.0 - kEps);
    if (clip && b1 > 0) r.hi = std::min(r.hi, (L - b1 - 1.0) * inv_s2 - 0.5 - 2 * kEps);
    if (clip && b2 > 0) r.lo = std::max(r.lo, -(L - b2 - 1.0) * inv_s2 + 0.5 + 2 * kEps);
    return r;
}

static int row_count(const Row& r) { return (int)std::floor((r.hi - r.lo) / (1.0 + kEps)) + 1; }

// The squares of a row, centred on the row's v-range.
static void emit_row(std::vector<Pt>& out, double u, const Row& r) {
    const double inv_s2 = 1.0 / std::sqrt(2.0), pi4 = std::acos(-1.0) * 0.25;
    const int cnt = row_count(r);
    const double span = (cnt - 1) * (1.0 + kEps);
    const double v0 = 0.5 * (r.lo + r.hi) - 0.5 * span;
    for (int m = 0; m < cnt; ++m) {
        const double v = v0 + m * (1.0 + kEps);
        out.push_back({(u - v) * inv_s2, (u + v) * inv_s2, pi4});
    }
}

// A corner triangle of `a` unit squares (rows of a, a-1, ..., 1).
static void emit_corner(std::vector<Pt>& out, int a, double L, bool right, bool top) {
    for (int i = 0; i < a; ++i)
        for (int j = 0; i + j < a; ++j)
            out.push_back({right ? L - 0.5 - i - kEps : 0.5 + i + kEps, top ? L - 0.5 - j - kEps : 0.5 + j + kEps, 0.0});
}

static std::vector<Topo> topologies(int n, double seed_L) {
    const double inv_s2 = 1.0 / std::sqrt(2.0);
    std::vector<Topo> cands;
    for (int w = 1; w <= 24; ++w) {
        for (int a1 = 0; a1 <= 32; ++a1) {
            for (int a2 = a1; a2 <= 32; ++a2) {
                const double L = 0.5 * (a1 + a2) + 1.0 + w * inv_s2 + (w + 4) * kEps;
                if (L < std::sqrt((double)n) - 0.05 || L > seed_L + 0.15) continue;
                const double u0 = (a1 + 1.0) * inv_s2 + 0.5 + 2 * kEps;
                const int b_lim = (int)std::floor(L - std::max(a1, a2));
                for (int b1 = 0; b1 <= std::max(0, b_lim); ++b1) {
                    for (int b2 = 0; b2 <= b1; ++b2) {
                        const int corner_cnt = a1 * (a1 + 1) / 2 + a2 * (a2 + 1) / 2 + b1 * (b1 + 1) / 2 + b2 * (b2 + 1) / 2;
                        if (corner_cnt > n + 3) continue;
                        int band_cnt = 0;
                        for (int k = 0; k < w; ++k) {
                            const Row r = band_row(u0 + k * (1.0 + kEps), L, b1, b2, true);
                            if (r.hi >= r.lo) band_cnt += row_count(r);
                        }
                        const int cap = corner_cnt + band_cnt;
                        if (cap < n || cap > n + 4) continue;
                        std::vector<Pt> corners, band;
                        emit_corner(corners, a1, L, false, false);
                        emit_corner(corners, a2, L, true, true);
                        emit_corner(corners, b1, L, false, true);
                        emit_corner(corners, b2, L, true, false);
                        for (int k = 0; k < w; ++k) {
                            const double u = u0 + k * (1.0 + kEps);
                            const Row r = band_row(u, L, b1, b2, true);
                            if (r.hi >= r.lo) emit_row(band, u, r);
                        }
                        // corners first, then the band (and, with spare room, the band first)
                        std::vector<Pt> pts = corners;
                        for (size_t t = 0; t < band.size() && (int)pts.size() < n; ++t) pts.push_back(band[t]);
                        pts.resize((size_t)n);
                        cands.push_back({L, pts});
                        if (cap > n && !corners.empty()) {
                            std::vector<Pt> alt = band;
                            for (size_t t = 0; t < corners.size() && (int)alt.size() < n; ++t) alt.push_back(corners[t]);
                            alt.resize((size_t)n);
                            cands.push_back({L, alt});
                        }
                    }
                }
                // an unclipped band one or two squares short: corner squares fill in
                std::vector<Pt> pts;
                emit_corner(pts, a1, L, false, false);
                emit_corner(pts, a2, L, true, true);
                for (int k = 0; k < w; ++k) {
                    const double u = u0 + k * (1.0 + kEps);
                    const Row r = band_row(u, L, 0, 0, false);
                    if (r.hi >= r.lo) emit_row(pts, u, r);
                }
                if ((int)pts.size() == n - 1 && L > std::max(a1, a2) + 1.0) {
                    pts.push_back({0.5 + kEps, L - 0.5 - kEps, 0.0});
                    cands.push_back({L + 0.005, pts});
                } else if ((int)pts.size() == n - 2 && L > std::max(a1, a2) + 1.0) {
                    pts.push_back({0.5 + kEps, L - 0.5 - kEps, 0.0});
                    pts.push_back({L - 0.5 - kEps, 0.5 + kEps, 0.0});
                    cands.push_back({L + 0.01, pts});
                }
            }
        }
    }
    std::sort(cands.begin(), cands.end(), [](const Topo& a, const Topo& b) { return a.L < b.L; });
    if (cands.size() > 64) cands.resize(64);
    return cands;
}

// Groups 5-6: a corner grid, anchors, two tilted edge rows.
static std::vector<Pt> corner_grid(int n, double seed_L, int b) {
    const int group = b % 8, k_floor = (int)std::floor(std::sqrt((double)n));
    const int cx = std::max(1, k_floor - 1 - ((b / 8) % 2));
    const int cy = std::max(1, k_floor - 1 - ((b / 16) % 2));
    const bool cut = group == 6 && cx >= 2 && cy >= 2;
    const double Lb = std::max(std::sqrt((double)n) + 0.05, seed_L - 0.03);
    std::vector<Pt> pts;
    for (int i = 0; i < cx && (int)pts.size() < n; ++i)
        for (int j = 0; j < cy && (int)pts.size() < n; ++j) {
            if (cut && i == cx - 1 && j == cy - 1) continue;
            pts.push_back({0.5 + i, 0.5 + j, 0.0});
        }
    if (((b / 8) % 3) != 0 && (int)pts.size() < n) pts.push_back({Lb - 0.5, Lb - 0.5, 0.0});
    if (((b / 8) % 3) == 1 && (int)pts.size() < n) {
        pts.push_back({0.5, Lb - 0.5, 0.0});
        if ((int)pts.size() < n) pts.push_back({Lb - 0.5, 0.5, 0.0});
    }
    const double th = 0.25 + 0.08 * ((b / 8) % 7);
    const int rem = n - (int)pts.size();
    const int n_right = (rem + 1) / 2, n_top = rem - n_right;
    for (int k = 0; k < n_right; ++k) {
        const double y = 0.7 + (Lb - 1.4) * (k + 0.5) / std::max(1, n_right);
        const double x = 0.5 * (cx + Lb) + ((k % 2 == 0) ? -0.18 : 0.18);
        pts.push_back({std::clamp(x, 0.6, Lb - 0.6), std::clamp(y, 0.6, Lb - 0.6), th});
    }
    for (int k = 0; k < n_top; ++k) {
        const double x = 0.7 + (Lb - 1.4) * (k + 0.5) / std::max(1, n_top);
        const double y = 0.5 * (cy + Lb) + ((k % 2 == 0) ? -0.18 : 0.18);
        pts.push_back({std::clamp(x, 0.6, Lb - 0.6), std::clamp(y, 0.6, Lb - 0.6), th});
    }
    return pts;
}

// Group 7: four corner anchors and a rotated grid of the rest.
static std::vector<Pt> anchored_grid(int n, double seed_L, int b) {
    const double Lb = std::max(std::sqrt((double)n) + 0.05, seed_L - 0.02);
    std::vector<Pt> pts;
    pts.push_back({0.5, 0.5, 0.0});
    if (n > 1) pts.push_back({Lb - 0.5, 0.5, 0.0});
    if (n > 2) pts.push_back({0.5, Lb - 0.5, 0.0});
    if (n > 3) pts.push_back({Lb - 0.5, Lb - 0.5, 0.0});
    const int rem = n - (int)pts.size();
    const int cols = std::max(1, (int)std::ceil(std::sqrt((double)rem)));
    const double th = 0.35 + 0.07 * ((b / 8) % 6);
    for (int k = 0; k < rem; ++k) {
        const int ix = k % cols, iy = k / cols;
        pts.push_back({0.8 + (Lb - 1.6) * (ix + 0.5) / cols, 0.8 + (Lb - 1.6) * (iy + 0.5) / cols, th});
    }
    return pts;
}

static uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static double unit(uint64_t& s) {  // uniform in [0, 1)
    s = mix64(s);
    return (double)(s >> 11) * (1.0 / 9007199254740992.0);
}
static double wrap_quarter(double a) {
    const double q = 1.5707963267948966;
    a = std::fmod(a, q);
    return a < 0.0 ? a + q : a;
}

}  // namespace port
}  // namespace sqs

using namespace sqs;
using namespace sqs::port;

extern "C" int sqs_portfolio(int n, double L, const double* seed_xya, int chains, int structured, uint64_t rng_seed,
                             int jitter, double* out) {
    SQS_REQUIRE(n >= 1 && n <= 1000, "n=%d out of 1..1000", n);
    SQS_REQUIRE(chains >= 1 && chains <= 4096, "chains=%d out of 1..4096", chains);
    SQS_REQUIRE(std::isfinite(L) && L > 0 && L <= 64, "L must be in (0, 64]");
    SQS_REQUIRE(seed_xya && out, "null pointer");
    for (int b = 0; b < chains; ++b) std::memcpy(out + 3 * (size_t)b * n, seed_xya, sizeof(double) * 3 * n);
    if (!structured || n <= 1) return SQS_OK;
    const std::vector<Topo> cands = topologies(n, L);
    for (int b = 0; b < chains; ++b) {
        const int ladder = b / 8, group = b % 8;
        std::vector<Pt> pts;
        if (group <= 1) {
            if (ladder >= 2 && !cands.empty()) pts = cands[(size_t)(ladder - 2) % cands.size()].pts;
        } else if (group <= 4 && !cands.empty()) {
            pts = cands[(size_t)ladder % cands.size()].pts;
        } else if (group == 5 || group == 6) {
            pts = corner_grid(n, L, b);
        } else {
            pts = anchored_grid(n, L, b);
        }
        double* dst = out + 3 * (size_t)b * n;
        for (size_t i = 0; i < pts.size() && (int)i < n; ++i) {
            dst[3 * i] = pts[i].x;
            dst[3 * i + 1] = pts[i].y;
            dst[3 * i + 2] = pts[i].a;
        }
        if (!jitter || group == 0) continue;
        uint64_t s = rng_seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(b + 1));
        const double amp = group == 1 ? 1e-4 * std::pow(100.0, unit(s)) : 0.03;
        for (int i = 0; i < n; ++i) {
            dst[3 * i] = std::fmin(L - 0.5, std::fmax(0.5, dst[3 * i] + amp * (2.0 * unit(s) - 1.0)));
            dst[3 * i + 1] = std::fmin(L - 0.5, std::fmax(0.5, dst[3 * i + 1] + amp * (2.0 * unit(s) - 1.0)));
            dst[3 * i + 2] = wrap_quarter(dst[3 * i + 2] + amp * (2.0 * unit(s) - 1.0));
        }
    }
    return SQS_OK;
}
