// Native check of the task builder (built and run by tests/test_tasks_cpu.py):
// for every device phase of the rules, in several modes (batch tasks with
// the default settings; every phase walked and split into tiny tasks; one
// rule at a time as the per-rule calls build them), the tasks must
//   * cover every root of the phase exactly once: by one plain task, or by
//     the slices of a split root, which partition its first segment in order;
//   * hold at most the plan's group of roots per plain task (the size its
//     dedup bitmap is laid out for);
//   * give every split root its own global row, numbered 0 .. heavyRows-1.
// It also checks the chained fan-out (TaskBuilder::transition) of every pair
// of consecutive expand steps against a direct mean over the first step's
// edges, capped and uncapped.
// Usage: tasks_check GRAPH.ttl RULES.txt
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <map>
#include <string>
#include <vector>

#include "../../masterthesis_gpu_acceleration_b200/csrc/index.hpp"
#include "../../masterthesis_gpu_acceleration_b200/csrc/planner.hpp"
#include "../../masterthesis_gpu_acceleration_b200/csrc/rules.hpp"
#include "../../masterthesis_gpu_acceleration_b200/csrc/tasks.hpp"
#include "../../masterthesis_gpu_acceleration_b200/csrc/turtle.hpp"

using namespace gr;

namespace {

long check_phase(TaskBuilder& tb, const PhasePlan& ph, const PhaseTasks& pt, int idx) {
    long bad = 0;
    const DevPlan& P = ph.plan;
    const int32_t R = ph.rootEnd - ph.rootBeg;
    int32_t g = std::max(P.groupMax, 1);
    if (ph.needsGlobalBitmap) g = std::min(P.cap, 512);
    std::vector<int> cover((size_t)std::max(R, 0), 0);
    std::map<int32_t, std::vector<const DevTask*>> slices;   // split root -> its slices
    std::map<int32_t, int32_t> rowOf;                        // split root -> global row
    if (pt.cost.size() != pt.tasks.size()) ++bad;
    for (const DevTask& t : pt.tasks) {
        if (t.plan != idx || t.beg < ph.rootBeg || t.end > ph.rootEnd || t.beg >= t.end) { ++bad; continue; }
        if (t.gRow < 0) {
            if (t.end - t.beg > g) ++bad;
            for (int32_t r = t.beg; r < t.end; ++r) ++cover[(size_t)(r - ph.rootBeg)];
        } else {
            if (t.end != t.beg + 1 || t.gRow >= pt.heavyRows) { ++bad; continue; }
            slices[t.beg].push_back(&t);
            auto it = rowOf.emplace(t.beg, t.gRow).first;
            if (it->second != t.gRow) ++bad;
        }
    }
    std::vector<int> rowUse((size_t)std::max(pt.heavyRows, 0), 0);
    for (auto& kv : slices) {
        const int32_t r = kv.first;
        ++cover[(size_t)(r - ph.rootBeg)];
        ++rowUse[(size_t)rowOf[r]];
        int32_t vals[2];
        tb.root_vals(P, r, vals);
        const auto seg = tb.first_segment(P, r, vals);
        int32_t at = 0;
        for (const DevTask* t : kv.second) {   // slices appear in order
            if (t->sub0 != at || t->sub1 <= t->sub0) ++bad;
            at = t->sub1;
        }
        if (at != seg.second - seg.first || kv.second.size() < 2) ++bad;
    }
    for (int c : cover) if (c != 1) ++bad;
    for (int u : rowUse) if (u != 1) ++bad;
    return bad;
}

// Mean row length under (p1, d1) of val[d0][e] over every edge e of p0,
// straight from the edge arrays.
double direct_transition(const HostIndex& ix, int32_t p0, int d0, int32_t p1, int d1, bool capped) {
    double n = 0, acc = 0;
    for (int32_t r = ix.predRow[d0][p0]; r < ix.predRow[d0][p0 + 1]; ++r)
        for (int32_t e = ix.rowBeg[d0][r]; e < ix.rowBeg[d0][r + 1]; ++e) {
            const auto rr = ix.row_range(p1, d1, ix.val[d0][e]);
            double d = rr.second - rr.first;
            if (capped) d = std::min(d, (double)kHubMinDegree);
            n += 1;
            acc += d;
        }
    return n > 0 ? acc / n : 0.0;
}

long check_transitions(TaskBuilder& tb, const HostIndex& ix, const DevPlan& P, size_t& checked) {
    long bad = 0;
    for (int s = 1; s < P.m; ++s) {
        const DevStep& a = P.steps[s - 1];
        const DevStep& b = P.steps[s];
        if (a.kind != kExpand || b.kind != kExpand) continue;
        for (bool capped : {false, true}) {
            const double got = tb.transition(a.pred, a.dir, b.pred, b.dir, capped);
            const double want = direct_transition(ix, a.pred, a.dir, b.pred, b.dir, capped);
            if (std::fabs(got - want) > 1e-9 * std::max(1.0, want)) ++bad;
            ++checked;
        }
    }
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
    std::vector<RulePlan> rps;
    Geom geom;
    while (std::getline(in, line)) {
        if (line.empty()) continue;
        try {
            rps.push_back(plan_rule(parser.parse_text(line), ix, geom));
        } catch (const RuleError&) {
        }
    }
    std::vector<const PhasePlan*> phases;
    for (const RulePlan& rp : rps) {
        if (rp.status != kRuleOk) continue;
        if (rp.support.how == kDevice) phases.push_back(&rp.support);
        if (rp.body.how == kDevice) phases.push_back(&rp.body);
    }
    const int blocks = 148 * (1024 / geom.block);
    long bad = 0;
    size_t tasks = 0, splitRoots = 0;
    auto run = [&](TaskBuilder& tb, const std::vector<const PhasePlan*>& ph, double budget, bool costAware) {
        std::vector<PhaseTasks> out;
        tb.build(ph, blocks, true, out, budget, costAware);
        if (out.size() != ph.size()) { ++bad; return; }
        for (size_t i = 0; i < ph.size(); ++i) {
            bad += check_phase(tb, *ph[i], out[i], (int)i);
            tasks += out[i].tasks.size();
            splitRoots += (size_t)out[i].heavyRows;
        }
    };
    {   // batch tasks, default settings
        TaskBuilder tb(ix);
        run(tb, phases, 4.0e7, false);
    }
    {   // every phase walked, tiny tasks: many split roots
        TaskBuilder tb(ix);
        tb.walkThreshold = 0;
        tb.forceTarget = 3;
        run(tb, phases, 1.0e12, false);
    }
    {   // one rule at a time, as per-rule calls build them
        TaskBuilder tb(ix);
        for (const RulePlan& rp : rps) {
            std::vector<const PhasePlan*> one;
            if (rp.status != kRuleOk) continue;
            if (rp.support.how == kDevice) one.push_back(&rp.support);
            if (rp.body.how == kDevice) one.push_back(&rp.body);
            if (!one.empty()) run(tb, one, 4.0e6, true);
        }
    }
    size_t transitions = 0;
    {   // chained fan-outs against the edge arrays
        TaskBuilder tb(ix);
        for (const PhasePlan* ph : phases) bad += check_transitions(tb, ix, ph->plan, transitions);
    }
    std::printf("phases %zu tasks %zu split roots %zu transitions %zu violations %ld\n", phases.size(), tasks,
                splitRoots, transitions, bad);
    return bad == 0 ? 0 : 1;
}
