// TEST INFRASTRUCTURE ONLY -- the host-side portfolio builder of the
// reference's `packing` program (dpack::build_portfolio, packing.cu), compiled
// from the reference source where it lies into oracle/_ref/libref_packing.so
// so tests can compare the library's portfolio with it.  Not shipped.
#define main sqs_reference_packing_main
#include "packing.cu"
#undef main

extern "C" int ref_build_portfolio_packing(int n, int chains, double L, const double* seed_xya, double* out) {
    std::vector<dpack::P> seed((size_t)n), h;
    for (int i = 0; i < n; ++i) seed[(size_t)i] = dpack::P{seed_xya[3 * i], seed_xya[3 * i + 1], seed_xya[3 * i + 2]};
    dpack::build_portfolio(n, chains, L, seed, h);
    for (size_t k = 0; k < h.size(); ++k) {
        out[3 * k] = h[k].x;
        out[3 * k + 1] = h[k].y;
        out[3 * k + 2] = h[k].a;
    }
    return (int)h.size();
}
