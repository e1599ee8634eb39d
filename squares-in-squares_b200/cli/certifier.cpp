// Drop-in for the reference's certifier program (certifier.cpp:933-1077):
//
//   certifier <submission.csv> [--max-n N] [--threads T] [--roundtrip] [--details out.json]
//
// Same CSV rules (header "id,n,square_id,x,y,angle", consecutive ids from 0,
// six fields per row, 1 <= n <= 1000; a violation exits 2), rows of every
// n <= max_n form that n's packing in file order, a missing n scores the
// grid penalty with reason "missing from submission", and the same summary
// line on stdout and per-n details file.  All packings are certified in one
// sqs_certify_batch call on the GPU, whose verdicts, reasons, scores and
// 50-decimal sides equal the reference's evaluate_single_puzzle; --roundtrip
// applies the same literal transform there.  --threads is accepted and
// reported (the GPU batch does not use host threads).  Caller:
// cpp_loop.gates (cuda/cpp_loop.py:17-28).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <thread>
#include <vector>

#include "sqs.h"

namespace {

struct Row {
    int sid;
    std::string x, y, a;
};

// Score of a missing packing: the ceil(sqrt n) grid's side over the area
// bound sqrt n, minus 1 (infeasible_score, certifier.cpp:734-736).
double grid_penalty(int n) {
    const double s = std::ceil(std::sqrt((double)n));
    return s / std::sqrt((double)n) - 1.0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::cerr << "Usage: certifier <submission.csv> [--max-n N] [--threads T] [--roundtrip] [--details out.json]\n";
        return 2;
    }
    const std::string csv_path = argv[1];
    int max_n = 1000;
    int threads = (int)std::max(1u, std::thread::hardware_concurrency());
    bool roundtrip = false;
    std::string details;
    for (int i = 2; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "--max-n" && i + 1 < argc) max_n = std::atoi(argv[++i]);
        else if (a == "--threads" && i + 1 < argc) threads = std::max(1, std::atoi(argv[++i]));
        else if (a == "--roundtrip") roundtrip = true;
        else if (a == "--details" && i + 1 < argc) details = argv[++i];
    }
    const auto t0 = std::chrono::steady_clock::now();
    std::ifstream in(csv_path);
    if (!in) {
        std::cerr << "Cannot open " << csv_path << "\n";
        return 2;
    }
    std::string line;
    if (!std::getline(in, line)) {
        std::cerr << "Empty CSV\n";
        return 2;
    }
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line != "id,n,square_id,x,y,angle") {
        std::cerr << "CSV header must be id,n,square_id,x,y,angle\n";
        return 2;
    }
    const int top = std::max(0, max_n);
    std::vector<std::vector<Row>> puzzles((size_t)top + 1);
    long long expected = 0;
    while (std::getline(in, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        if (line.empty()) continue;
        size_t c[5];
        size_t from = 0;
        for (int k = 0; k < 5; ++k) {
            c[k] = line.find(',', from);
            if (c[k] == std::string::npos) return 2;
            from = c[k] + 1;
        }
        if (line.find(',', c[4] + 1) != std::string::npos) return 2;
        const long long id = std::strtoll(line.c_str(), nullptr, 10);
        if (id != expected) {
            std::cerr << "Row id mismatch at " << expected << "\n";
            return 2;
        }
        ++expected;
        const int n = std::atoi(line.c_str() + c[0] + 1);
        const int sid = std::atoi(line.c_str() + c[1] + 1);
        if (n < 1 || n > 1000) return 2;
        if (n <= max_n)
            puzzles[(size_t)n].push_back(Row{sid, line.substr(c[2] + 1, c[3] - c[2] - 1),
                                             line.substr(c[3] + 1, c[4] - c[3] - 1), line.substr(c[4] + 1)});
    }

    // one batch: every present n
    std::vector<int32_t> n_of, sid;
    std::vector<int64_t> row_start{0}, lit_off{0};
    std::string text;
    std::vector<int> which;
    for (int n = 1; n <= max_n; ++n) {
        if (puzzles[(size_t)n].empty()) continue;
        which.push_back(n);
        n_of.push_back(n);
        for (const Row& r : puzzles[(size_t)n]) {
            sid.push_back(r.sid);
            for (const std::string* s : {&r.x, &r.y, &r.a}) {
                text += *s;
                lit_off.push_back((int64_t)text.size());
            }
        }
        row_start.push_back(row_start.back() + (int64_t)puzzles[(size_t)n].size());
    }
    std::vector<sqs_verdict> ver(which.size());
    if (!which.empty()) {
        sqs_ctx* ctx = nullptr;
        if (sqs_ctx_create(0, &ctx) != SQS_OK ||
            sqs_certify_batch(ctx, (int)which.size(), n_of.data(), row_start.data(), sid.data(),
                              text.empty() ? "" : text.data(), lit_off.data(), roundtrip ? SQS_CERT_ROUNDTRIP : 0,
                              ver.data()) != SQS_OK) {
            std::cerr << "certifier: " << sqs_last_error() << "\n";
            return 2;
        }
        sqs_ctx_destroy(ctx);
    }
    struct Res {
        double score;
        bool ok;
        std::string L, reason;
    };
    std::vector<Res> res((size_t)top + 1);
    for (int n = 1; n <= max_n; ++n) res[(size_t)n] = Res{grid_penalty(n), false, "", "missing from submission"};
    for (size_t k = 0; k < which.size(); ++k)
        res[(size_t)which[k]] = Res{ver[k].score, ver[k].ok != 0, ver[k].L, ver[k].reason};

    double total = 0.0;
    int accepted = 0, missing = 0, rejected = 0;
    for (int n = 1; n <= max_n; ++n) {
        total += res[(size_t)n].score;
        if (res[(size_t)n].ok) ++accepted;
        else if (res[(size_t)n].reason == "missing from submission") ++missing;
        else ++rejected;
    }
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    auto head = [&](std::ostream& o) {
        o << std::setprecision(17) << "{\"score\":" << total << ",\"max_n\":" << max_n << ",\"accepted\":" << accepted
          << ",\"missing\":" << missing << ",\"rejected\":" << rejected << ",\"seconds\":" << sec
          << ",\"threads\":" << threads << ",\"roundtrip\":" << (roundtrip ? "true" : "false");
    };
    if (!details.empty()) {
        std::ofstream out(details);
        head(out);
        out << ",\"results\":[";
        for (int n = 1; n <= max_n; ++n) {
            const Res& r = res[(size_t)n];
            if (n > 1) out << ",";
            out << "{\"n\":" << n << ",\"score\":" << r.score << ",\"L\":" << (r.ok ? "\"" + r.L + "\"" : "null")
                << ",\"reason\":\"" << r.reason << "\"}";
        }
        out << "]}\n";
    }
    head(std::cout);
    std::cout << "}\n";
    return 0;
}
