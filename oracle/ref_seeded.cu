// TEST INFRASTRUCTURE ONLY -- builds the reference's own FP64 energy
// functions (seeded.cu:41-113, compiled from the reference source where it
// lies) into oracle/_ref/libref_seeded.so so tests can pin the oracle
// restatement and bench.py can time the reference's CPU path.  Not shipped.
#define main sqs_reference_seeded_main
#include "seeded.cu"
#undef main
#include <thread>

extern "C" double ref_pair(const double* p, const double* q, double* g) {
    P a{p[0], p[1], p[2]}, b{q[0], q[1], q[2]};
    if (!g) return pair(a, b);
    G gg{g[0], g[1], g[2]};
    double e = pair(a, b, &gg);
    g[0] = gg.x; g[1] = gg.y; g[2] = gg.a;
    return e;
}

extern "C" double ref_pair_smooth(const double* p, const double* q, double* g) {
    P a{p[0], p[1], p[2]}, b{q[0], q[1], q[2]};
    G gg{g[0], g[1], g[2]};
    double e = pair_cached_smooth(a, b, cos(a.a), sin(a.a), cos(b.a), sin(b.a), &gg);
    g[0] = gg.x; g[1] = gg.y; g[2] = gg.a;
    return e;
}

extern "C" double ref_boundary(const double* p, double L, double* g) {
    P a{p[0], p[1], p[2]};
    if (!g) return boundary(a, L);
    G gg{g[0], g[1], g[2]};
    double e = boundary(a, L, &gg);
    g[0] = gg.x; g[1] = gg.y; g[2] = gg.a;
    return e;
}

// Energy = sum boundary + sum_{i<j} pair; gradient_i = d boundary_i +
// sum_{j != i} d pair(p_i, p_j)/d p_i -- the reference's own all-pairs CPU
// path, built only from its pair()/boundary().
static double ref_total_one(int n, double L, const double* xya, double* grad) {
    double e = 0.0;
    for (int i = 0; i < n; ++i) {
        P p{xya[3 * i], xya[3 * i + 1], xya[3 * i + 2]};
        G g{0, 0, 0};
        e += boundary(p, L, grad ? &g : nullptr);
        for (int j = 0; j < n; ++j) {
            if (j == i) continue;
            P q{xya[3 * j], xya[3 * j + 1], xya[3 * j + 2]};
            if (j > i) e += pair(p, q, grad ? &g : nullptr);
            else if (grad) pair(p, q, &g);
        }
        if (grad) { grad[3 * i] = g.x; grad[3 * i + 1] = g.y; grad[3 * i + 2] = g.a; }
    }
    return e;
}

extern "C" int ref_total_batch(int configs, int n, const double* xya, const double* L,
                               double* energy, double* grad, int threads) {
    if (threads < 1) threads = 1;
    if (threads > configs) threads = configs > 0 ? configs : 1;
    std::vector<std::thread> pool;
    auto work = [&](int t) {
        int a = (int)((long long)configs * t / threads), b = (int)((long long)configs * (t + 1) / threads);
        for (int c = a; c < b; ++c) {
            size_t off = (size_t)c * 3 * n;
            energy[c] = ref_total_one(n, L[c], xya + off, grad ? grad + off : nullptr);
        }
    };
    for (int t = 1; t < threads; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto& th : pool) th.join();
    return threads;
}

// The reference's structured initial portfolio (build_portfolio, host code
// in seeded.cu) for `chains` chains: out[b][i] = (x, y, angle), before the
// device-side jitter of structured_init.
extern "C" int ref_build_portfolio(int n, int chains, double L, const double* seed_xya, int structured,
                                   double* out) {
    std::vector<P> seed((size_t)n), h;
    for (int i = 0; i < n; ++i) seed[(size_t)i] = P{seed_xya[3 * i], seed_xya[3 * i + 1], seed_xya[3 * i + 2]};
    build_portfolio(n, chains, L, seed, structured, 0ull, h);
    for (size_t k = 0; k < h.size(); ++k) {
        out[3 * k] = h[k].x;
        out[3 * k + 1] = h[k].y;
        out[3 * k + 2] = h[k].a;
    }
    return (int)h.size();
}
