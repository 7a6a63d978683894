// planner.hpp — rule -> device plans (support phase and body-size phase).
#pragma once
#include <cstdint>
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
};

// Plans both phases.  Semantics follow CPU_01_nonparallel/SupportCounting.cpp:
// support (474-552) with the head triple counted as used, body size
// (563-631) with the seed atom's keys as headS candidates.
RulePlan plan_rule(const Rule& rule, const HostIndex& ix, const Geom& geom);

}  // namespace gr
