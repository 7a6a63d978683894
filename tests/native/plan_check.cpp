// Native check of the planner's shared-memory layout (built and run by
// tests/test_plan_cpu.py): for every device phase of the rules, planned for
// 128-, 256- and 512-thread blocks, the frontier levels end at or before the
// dedup bitmap, the bitmap holds the widest task the plan allows, the
// capacity is a positive multiple of 32, and every index a plan holds (tuple
// positions, check and used-triple ranges, constants) stays inside its
// arrays.  The kernel indexes its shared pool by these fields unchecked.
// Usage: plan_check GRAPH.ttl RULES.txt
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "../../masterthesis_gpu_acceleration_b200/csrc/index.hpp"
#include "../../masterthesis_gpu_acceleration_b200/csrc/planner.hpp"
#include "../../masterthesis_gpu_acceleration_b200/csrc/rules.hpp"
#include "../../masterthesis_gpu_acceleration_b200/csrc/turtle.hpp"

using namespace gr;

namespace {

bool ref_ok(TermRef r, int len, int nConsts) {
    return r < 0 ? (-1 - r) < nConsts : (r >= 0 && r < len);
}

long check_plan(const PhasePlan& ph, const Geom& geom) {
    long bad = 0;
    const DevPlan& P = ph.plan;
    const int pool = geom.poolInts();
    if (P.m < 0 || P.m > kMaxBody) return 1;
    if (P.cap < 32 || P.cap % 32 != 0) ++bad;
    int end = 0;   // end of the frontier levels in the pool
    if (P.m == 0) end = P.cap * P.tupleLen[0];
    for (int l = 0; l < P.m; ++l) end += P.cap * (P.tupleLen[l] + 2);
    if (end > P.bitmapOff || P.bitmapOff > pool) ++bad;
    // the task's shared dedup bits: found bits of up to groupMax roots, or
    // groupMax pair rows when the pair bitmap is local
    const int rowWords = P.mode == kPairs ? std::max(1, (P.wo + 31) / 32) : 1;
    const long need = P.mode == kPairs ? (ph.needsGlobalBitmap ? 0 : (long)P.groupMax * rowWords)
                                       : (long)(P.groupMax + 31) / 32;
    if (P.bitmapOff + need > pool) ++bad;
    if (P.groupMax < 1 || P.groupMax > P.cap) ++bad;
    const int nConsts = kMaxConsts;   // constant references index the fixed-size consts[]
    for (int l = 0; l <= P.m; ++l) {
        if (P.tupleLen[l] < kTupleHead || P.tupleLen[l] > kMaxTuple) ++bad;
        if (l > 0 && P.tupleLen[l] != P.tupleLen[l - 1] + P.steps[l - 1].nNew) ++bad;
        if (P.chkBeg[l] < 0 || P.chkN[l] < 0 || P.chkBeg[l] + P.chkN[l] > kMaxChecks) ++bad;
        if (P.usedBeg[l] < 0 || P.usedN[l] < 0 || P.usedBeg[l] + P.usedN[l] > kMaxUsed) ++bad;
        for (int c = P.chkBeg[l]; c < P.chkBeg[l] + P.chkN[l] && c < kMaxChecks; ++c) {
            const DevCheck& C = P.checks[c];
            if (!ref_ok(C.s, P.tupleLen[l], nConsts) || !ref_ok(C.o, P.tupleLen[l], nConsts)) ++bad;
        }
        for (int u = P.usedBeg[l]; u < P.usedBeg[l] + P.usedN[l] && u < kMaxUsed; ++u) {
            const DevUsed& U = P.used[u];
            for (TermRef r : {U.sA, U.oA, U.sB, U.oB})
                if (!ref_ok(r, P.tupleLen[l], nConsts)) ++bad;
        }
    }
    for (int s = 0; s < P.m; ++s) {
        const DevStep& st = P.steps[s];
        if (st.nNew < 1 || st.nNew > 2) ++bad;
        if (st.kind == kExpand && !ref_ok(st.keyRef, P.tupleLen[s], nConsts)) ++bad;
    }
    if (P.mode == kPairs && (P.hoLevel < 1 || P.hoLevel > P.m)) ++bad;
    return bad;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    std::string text, err;
    if (!read_file(argv[1], text, &err)) { std::fprintf(stderr, "%s\n", err.c_str()); return 2; }
    TermDict ents, preds;
    std::vector<int32_t> spo;
    parse_turtle_text(text, ents, preds, spo);
    HostIndex ix = build_index(spo, (int32_t)ents.size(), (int32_t)preds.size(), kHubMinDegree);
    RuleParser parser(ents, preds, scan_rule_prefixes_text(text));
    std::ifstream in(argv[2]);
    std::string line;
    std::vector<Rule> rules;
    while (std::getline(in, line)) {
        if (line.empty()) continue;
        try {
            rules.push_back(parser.parse_text(line));
        } catch (const RuleError&) {
        }
    }
    long bad = 0, phases = 0;
    for (int block : {128, 256, 512}) {
        Geom geom;
        geom.block = block;
        for (const Rule& r : rules) {
            const RulePlan rp = plan_rule(r, ix, geom);
            if (rp.status != kRuleOk) continue;
            for (const PhasePlan* ph : {&rp.support, &rp.body})
                if (ph->how == kDevice) {
                    ++phases;
                    bad += check_plan(*ph, geom);
                }
        }
    }
    std::printf("rules %zu device phases %ld violations %ld\n", rules.size(), phases, bad);
    return bad == 0 ? 0 : 1;
}
