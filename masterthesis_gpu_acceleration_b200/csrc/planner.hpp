// planner.hpp — rule -> device plans (support phase and body-size phase).
#pragma once
#include <cstdint>
#include <utility>
#include <vector>

#include "common.hpp"
#include "index.hpp"
#include "rules.hpp"

namespace gr {

enum RuleStatus : int32_t {
    kRuleOk = 0,
    kRuleUnsupported = 1,   // more than 8 body atoms, 16 variables or too many constants
};

// How a phase's count is obtained.
enum PhaseHow : int32_t {
    kStatic = 0,      // known on the host (value in `value`)
    kDevice = 1,      // plan + tasks on the device
};

struct PhasePlan {
    int32_t how = kStatic;
    int64_t value = 0;
    DevPlan plan{};
    int32_t rootBeg = 0, rootEnd = 0;   // root range (edges or rows)
    bool needsGlobalBitmap = false;     // kPairs whose hO domain exceeds the shared bitmap
    double estCost = 0.0;               // autotuner estimate (relative units)
};

struct RulePlan {
    int32_t status = kRuleOk;
    int64_t headSize = 0, headSupport = 0;
    PhasePlan support, body;
    // >= 0 when the support is the number of head triples (hS, supFuse, hO),
    // hS != hO, among the body-size phase's (hS, hO) pairs: both head terms
    // are distinct variables and no body atom can ground to the head triple
    // (the support plan has no used-triple test), so a body-size plan that
    // keeps its pair rows can count the support too (fused support).
    int32_t supFuse = -1;
};

// Where a kPairs plan ranks hO: the rows of (pred, dir) in the returned
// pair (the step binding hO looks its value up there).
std::pair<int32_t, int32_t> ho_domain(const DevPlan& P);

// Plans both phases.  Semantics follow CPU_01_nonparallel/SupportCounting.cpp:
// support (474-552) with the head triple counted as used, body size
// (563-631) with the seed atom's keys as headS candidates.
RulePlan plan_rule(const Rule& rule, const HostIndex& ix, const Geom& geom);

}  // namespace gr
