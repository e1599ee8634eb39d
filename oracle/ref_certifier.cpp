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

#include <atomic>
#include <thread>

// Certify `count` packings with `threads` worker threads pulling packings from
// an atomic counter, as certifier.cpp's main does (:1011-1032).  Packing p
// has rows row_start[p] .. row_start[p+1]-1; row r's literals are
// text[lit_off[3r+k] .. lit_off[3r+k+1]).  ok_out[p] = 1 when accepted.
// The same with each packing's 50-decimal side and reason written to
// L_out + 80 p and reason_out + 112 p (either may be NULL).
extern "C" int ref_evaluate_batch_text(int count, const int* n_of, const long long* row_start, const int* sid,
                                       const char* text, const long long* lit_off, int threads, int* ok_out,
                                       double* score_out, char* L_out, char* reason_out);

extern "C" int ref_evaluate_batch(int count, const int* n_of, const long long* row_start, const int* sid,
                                  const char* text, const long long* lit_off, int threads, int* ok_out,
                                  double* score_out) {
    return ref_evaluate_batch_text(count, n_of, row_start, sid, text, lit_off, threads, ok_out, score_out, nullptr,
                                   nullptr);
}

extern "C" int ref_evaluate_batch_text(int count, const int* n_of, const long long* row_start, const int* sid,
                                       const char* text, const long long* lit_off, int threads, int* ok_out,
                                       double* score_out, char* L_out, char* reason_out) {
    std::atomic<int> next{0};
    auto work = [&]() {
        for (int p = next.fetch_add(1); p < count; p = next.fetch_add(1)) {
            std::vector<cert::RowData> rd;
            for (long long r = row_start[p]; r < row_start[p + 1]; ++r) {
                cert::RowData d;
                d.square_id = sid ? sid[r] : (int)(r - row_start[p]);
                d.x.assign(text + lit_off[3 * r], (size_t)(lit_off[3 * r + 1] - lit_off[3 * r]));
                d.y.assign(text + lit_off[3 * r + 1], (size_t)(lit_off[3 * r + 2] - lit_off[3 * r + 1]));
                d.angle.assign(text + lit_off[3 * r + 2], (size_t)(lit_off[3 * r + 3] - lit_off[3 * r + 2]));
                rd.push_back(std::move(d));
            }
            cert::PuzzleResult res = cert::evaluate_single_puzzle(n_of[p], rd);
            ok_out[p] = res.ok ? 1 : 0;
            if (score_out) score_out[p] = res.score;
            if (L_out) put(L_out + 80 * (size_t)p, 80, res.ok ? res.L : std::string());
            if (reason_out) put(reason_out + 112 * (size_t)p, 112, res.reason);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
    return threads;
}
