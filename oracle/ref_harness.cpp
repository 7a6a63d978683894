// ref_harness.cpp — drives the reference's own CPU_01_nonparallel code.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/build_ref.sh against the
// reference sources where they lie (it compiles FinalRule.cpp, RdfIndexes.cpp,
// RuleParser.cpp and SupportCounting.cpp of CPU_01_nonparallel; nothing is
// copied).  The binary lands in oracle/_ref/ and serves two purposes:
//   * pinning the C restatement (oracle/rules_oracle.c) to the reference's
//     own results on the same Turtle graph and rule file;
//   * the timed CPU baseline, run the way CPU_01_nonparallel/main.cpp:63-126
//     runs it (parseTurtleFile, RuleParser over the same file, then
//     countSupport + countBodySize per rule, std::chrono around each).
//
// Usage:
//   cpu01_harness <graph.ttl> <rules.txt|rules.json> [--threads K]
//                 [--first N] [--repeat R] [--quiet]
// Output (stdout): one JSON object per rule, then a summary object.  With
// --threads K > 1 the rules are spread over K threads (each rule is still
// evaluated by the reference's single-threaded code; rules are independent
// and SupportCounting only reads the shared index).

#include "FinalRule.hpp"
#include "RdfIndexes.hpp"
#include "RuleParser.hpp"
#include "SupportCounting.hpp"

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

using Clock = std::chrono::steady_clock;

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s graph.ttl rules [--threads K] [--first N] [--repeat R] [--quiet]\n", argv[0]);
        return 2;
    }
    std::string ttl = argv[1], rulesFile = argv[2];
    int threads = 1, first = -1, repeat = 1;
    bool quiet = false;
    for (int i = 3; i < argc; ++i) {
        std::string a = argv[i];
        if (a == "--threads" && i + 1 < argc) threads = std::atoi(argv[++i]);
        else if (a == "--first" && i + 1 < argc) first = std::atoi(argv[++i]);
        else if (a == "--repeat" && i + 1 < argc) repeat = std::atoi(argv[++i]);
        else if (a == "--quiet") quiet = true;
    }
    if (threads < 1) threads = 1;
    try {
        auto t0 = Clock::now();
        RdfIndexes indexes;
        if (!indexes.parseTurtleFile(ttl)) { std::fprintf(stderr, "cannot parse %s\n", ttl.c_str()); return 1; }
        RuleParser parser(indexes, ttl);
        bool isJson = rulesFile.size() >= 5 && rulesFile.substr(rulesFile.size() - 5) == ".json";
        std::vector<FinalRule> rules = isJson ? parser.parseJsonRuleFile(rulesFile) : parser.parseRuleFile(rulesFile);
        if (first >= 0 && (size_t)first < rules.size()) rules.resize(first);
        auto t1 = Clock::now();
        SupportCounting counter(indexes);
        size_t n = rules.size();
        std::vector<double> supMs(n), confMs(n);
        double wallMs = 0.0;
        for (int rep = 0; rep < repeat; ++rep) {
            std::atomic<size_t> next{0};
            auto work = [&]() {
                for (;;) {
                    size_t i = next.fetch_add(1);
                    if (i >= n) break;
                    auto a = Clock::now();
                    counter.countSupport(rules[i]);
                    auto b = Clock::now();
                    counter.countBodySize(rules[i]);
                    auto c = Clock::now();
                    supMs[i] = std::chrono::duration<double, std::milli>(b - a).count();
                    confMs[i] = std::chrono::duration<double, std::milli>(c - b).count();
                }
            };
            auto w0 = Clock::now();
            if (threads == 1) work();
            else {
                std::vector<std::thread> pool;
                for (int t = 0; t < threads; ++t) pool.emplace_back(work);
                for (auto& th : pool) th.join();
            }
            wallMs += std::chrono::duration<double, std::milli>(Clock::now() - w0).count();
        }
        if (!quiet) {
            for (size_t i = 0; i < n; ++i) {
                const auto& m = rules[i].measures;
                std::printf("{\"rule\": %zu, \"support\": %d, \"headSize\": %d, \"headSupport\": %d, "
                            "\"bodySize\": %d, \"headCoverage\": %.17g, \"confidence\": %.17g, "
                            "\"supportMs\": %.6f, \"confidenceMs\": %.6f}\n",
                            i, m.support, m.headSize, m.headSupport, m.bodySize, m.headCoverage,
                            m.confidence, supMs[i], confMs[i]);
            }
        }
        std::printf("{\"summary\": true, \"rules\": %zu, \"threads\": %d, \"repeat\": %d, "
                    "\"load_ms\": %.3f, \"eval_wall_ms\": %.3f}\n",
                    n, threads, repeat,
                    std::chrono::duration<double, std::milli>(t1 - t0).count(), wallMs);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ERROR: %s\n", e.what());
        return 1;
    }
}
