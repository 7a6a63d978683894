// tasks.hpp — splitting device phases into balanced tasks (the autotuner).
#pragma once
#include <cstdint>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "common.hpp"
#include "index.hpp"
#include "planner.hpp"

namespace gr {

struct PhaseTasks {
    std::vector<DevTask> tasks;
    std::vector<double> cost;   // estimated work per task
    int32_t heavyRows = 0;      // global dedup rows used by split roots
    double work = 0.0;          // estimated work of the whole phase
    double scale = 1.0;         // learned device ns per unit of work
};

// Builds tasks for a batch of phases.  Work is measured in candidate
// bindings.  Every phase gets a cheap estimate from average fan-outs and a
// hub-aware one from size-biased fan-outs (the degree of a row reached by
// following a random edge, sum(d^2)/sum(d)); the phases the hub-aware
// estimate ranks heaviest get an exact two-level walk per root (first
// segment, and the size of each child's next segment) within a per-batch
// budget, cached by plan signature.  Tasks then hold roots whose work sums to
// at most `target` (about 1/8 of a block's fair share of the batch); a root
// heavier than that is split into slices of its first segment, each a task
// of its own that deduplicates in a global row.
class TaskBuilder {
public:
    explicit TaskBuilder(const HostIndex& ix) : ix_(ix) {}

    // phases[i] is planned as plan number i.  blocks: resident blocks of the
    // launch.  split=false keeps every root in shared-memory tasks.
    void build(const std::vector<const PhasePlan*>& phases, int blocks, bool split,
               std::vector<PhaseTasks>& out);

    size_t cache_bytes() const { return cacheBytes_; }

    // Feedback from an instrumented run of tasks built by build(): taskNs
    // holds each task's start and end time.  Learns, per plan signature, the
    // device time per unit of estimated work, and marks plans whose slowest
    // task exceeded the balancing target for an exact per-root walk.
    void learn(const std::vector<const PhasePlan*>& phases, const std::vector<DevTask>& tasks,
               const std::vector<double>& cost, const unsigned long long* taskNs, int blocks);

    // Overrides: a fixed task work target (0 = automatic) and the hub-aware
    // estimate above which a phase is walked.
    double forceTarget = 0.0;
    double walkThreshold = 2.0e5;

private:
    const HostIndex& ix_;
    std::unordered_map<int64_t, std::vector<int32_t>> deg_;      // (pred, dir) -> degree by entity
    std::unordered_map<int64_t, double> sbFan_;                  // (pred, dir) -> size-biased fan-out
    std::unordered_map<std::string, std::vector<float>> walks_;  // plan signature -> per-root work
    std::unordered_map<std::string, double> calib_;             // plan signature -> ns per work unit
    std::unordered_map<std::string, bool> mustWalk_;            // plan signature -> walk next time
    double defaultCalib_ = 1.0;
    size_t cacheBytes_ = 0;

    const int32_t* degrees(int32_t pred, int dir);
    double sb_fan(int32_t pred, int dir);
    double avg_fan(const DevStep& st) const;
    double estimate(const PhasePlan& ph, bool hubAware);
    const std::vector<float>& walk(const PhasePlan& ph);
    double child_work(const DevPlan& P, const int32_t* rootVals, int32_t e, const int32_t* deg2, double tail) const;
    int root_vals(const DevPlan& P, int32_t r, int32_t* vals) const;
    std::pair<int32_t, int32_t> first_segment(const DevPlan& P, const int32_t* vals) const;
};

}  // namespace gr
