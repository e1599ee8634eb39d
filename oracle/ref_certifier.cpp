// TEST INFRASTRUCTURE ONLY -- builds the reference certifier (certifier.cpp,
// compiled from the reference source where it lies) into
// oracle/_ref/libref_certifier.so, exposing cert::evaluate_single_puzzle
// (certifier.cpp:738-912) and cert::roundtrip_float_str (:914-929) to the
// tests and to bench.py's reference arm.  Not shipped.
#define main sqs_reference_certifier_main
#include "certifier.cpp"
#undef main
#include <cstring>

namespace {
void put(char* dst, int cap, const std::string& s) {
    if (!dst || cap <= 0) return;
    size_t k = std::min((size_t)cap - 1, s.size());
    std::memcpy(dst, s.data(), k);
    dst[k] = 0;
}
}

// One packing: rows given as parallel arrays of square_id and literals.
// Returns 1 when accepted, 0 when rejected.
extern "C" int ref_evaluate(int n, int rows, const int* sid, const char* const* xs,
                            const char* const* ys, const char* const* as,
                            char* L_out, int L_cap, char* reason_out, int reason_cap,
                            double* score) {
    std::vector<cert::RowData> rd((size_t)rows);
    for (int i = 0; i < rows; ++i) rd[i] = cert::RowData{sid[i], xs[i], ys[i], as[i]};
    cert::PuzzleResult r = cert::evaluate_single_puzzle(n, rd);
    put(L_out, L_cap, r.ok ? r.L : std::string());
    put(reason_out, reason_cap, r.reason);
    if (score) *score = r.score;
    return r.ok ? 1 : 0;
}

extern "C" void ref_roundtrip(const char* s, char* out, int cap) {
    put(out, cap, cert::roundtrip_float_str(s));
}
