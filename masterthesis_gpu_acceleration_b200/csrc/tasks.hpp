// tasks.hpp — splitting device phases into balanced tasks (the autotuner).
#pragma once
#include <atomic>
#include <cstdint>
#include <memory>
#include <functional>
#include <shared_mutex>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "common.hpp"
#include "index.hpp"
#include "planner.hpp"

namespace gr {

// Per-phase limits of one build: at most `group` roots per task (0: the
// plan's own limit) and at most `maxHeavy` heavy roots split over tasks that
// share a global dedup row (-1: no limit; further heavy roots stay whole).
struct PhaseLimits {
    int32_t group = 0;
    int32_t maxHeavy = -1;
};

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
// Host time of one step of a per-root walk (ns), for the cost-aware mode.
constexpr double kWalkNsPerEdge = 8.0;

// The signature of a phase is the identity of its device computation: the
// plan without its per-launch fields, and its root range.  Phases with equal
// signatures produce equal counts.  phase_equal compares two signatures;
// phase_hash is a 64-bit hash of one (the key of the task builder's caches).
bool phase_equal(const PhasePlan& a, const PhasePlan& b);
uint64_t phase_hash(const PhasePlan& ph);

class TaskBuilder {
public:
    explicit TaskBuilder(const HostIndex& ix);

    // phases[i] is planned as plan number i.  blocks: resident blocks of the
    // launch.  split=false keeps every root in shared-memory tasks.
    // walkBudget: first-segment edges that may be newly walked (cached
    // walks and phases marked by learn() are not counted).
    // costAware: walk a phase only when its expected device time exceeds
    // the walk's own host time, and cut only roots above a block's fair
    // share of their phase (per-rule launches, where nothing overlaps).
    // limits (optional): one entry per phase.
    void build(const std::vector<const PhasePlan*>& phases, int blocks, bool split,
               std::vector<PhaseTasks>& out, double walkBudget = 4.0e6, bool costAware = false,
               const std::vector<PhaseLimits>* limits = nullptr);

    // Estimated candidate bindings of a phase (average fan-outs; exact first
    // two levels for chain-shaped plans rooted at the first step's rows).
    double work_estimate(const PhasePlan& ph) { return estimate2(ph); }
    // The hub-aware estimate: every expansion at the size-biased fan-out of
    // its (predicate, direction), i.e. as if each step landed where a random
    // edge lands (an upper-side estimate for rules through hub entities).
    double hub_estimate(const PhasePlan& ph) { return estimate(ph, true); }

    size_t cache_bytes() const { return cacheBytes_; }

    // Row length of every entity under (pred, dir), indexed by entity
    // (cached; safe to call from several threads).
    const int32_t* degrees(int32_t pred, int dir);

    // Estimated device time of a phase: learned ns per unit for plans seen
    // by learn(), otherwise the work estimate times the learned default
    // (1 ns per unit before any learning).
    double expected_ns(const PhasePlan& ph);

    // Feedback from an instrumented run of tasks built by build(): taskNs
    // holds each task's start and end time.  Learns, per plan signature, the
    // device time per unit of estimated work, and marks plans whose slowest
    // task exceeded the balancing target for an exact per-root walk.
    // weight: how far a learned figure moves toward this run's (1 replaces
    // it; the serving loop, learning from many small launches, uses less).
    // minWorstNs: slowest-task time below which no walk is requested.
    void learn(const std::vector<const PhasePlan*>& phases, const std::vector<DevTask>& tasks,
               const std::vector<double>& cost, const unsigned long long* taskNs, int blocks,
               double weight = 1.0, double minWorstNs = 0.0);

    // Boundaries of n contiguous slices of a device phase's roots with about
    // equal estimated work (per-root walk): slice k is [cut[k], cut[k+1]),
    // cut[0] = rootBeg, cut[n] = rootEnd.
    std::vector<int32_t> split_roots(const PhasePlan& ph, int n);

    // Suffix memos known to the context: per-row flags of (p1, d1) for the
    // memo of (p1, d1) -> (p2, d2), or with p3 >= 0 of the three-step suffix
    // (p1, d1) -> (p2, d2) -> (p3, d3), and its cost per item in work units,
    // or null.  Walks of plans that end in such a suffix weigh memoised
    // items by that cost instead of their enumeration.
    std::function<const std::vector<uint8_t>*(int, int, int, int, int, int, double*)> memoRows;

    // Overrides: a fixed task work target (0 = automatic) and the hub-aware
    // estimate above which a phase is walked.
    double forceTarget = 0.0;
    double walkThreshold = 2.0e5;

private:
    const HostIndex& ix_;
    std::unordered_map<int64_t, std::vector<int32_t>> deg_;      // (pred, dir) -> degree by entity
    // per pred * 2 + dir: deg_'s array once built (read without a lock), and
    // the size-biased fan-out (computed once, at construction)
    std::vector<std::atomic<const int32_t*>> degAt_;
    std::vector<double> sbFan_;
    // Per-root work, and its sum and maximum over blocks of kWalkBlock
    // roots, so that task building steps over runs of light roots a block
    // at a time.
    static constexpr int kWalkBlock = 16;
    struct Walk {
        std::vector<float> w;      // per-root work
        std::vector<double> bsum;  // per block of kWalkBlock roots (full blocks only)
        std::vector<float> bmax;
        double sum = 0.0;
    };
    std::unordered_map<uint64_t, Walk> walks_;                   // phase hash -> per-root work
    struct Hop2 {
        std::vector<float> perRow;   // per row of (p0, d0): sum over its edges of the next degree
        double total = 0.0;
    };
    // (p0, d0, p1, d1) -> two-hop sums, in shards with a lock each, so that
    // the threads estimating a batch's phases do not all take one lock
    static constexpr int kHop2Shards = 64;
    struct Hop2Shard {
        std::shared_mutex mu;
        std::unordered_map<uint64_t, Hop2> map;
    };
    std::unique_ptr<Hop2Shard[]> hop2_;
    // (p0, d0, p1, d1, capped) -> mean next degree per edge (see transition)
    struct TransShard {
        std::shared_mutex mu;
        std::unordered_map<uint64_t, double> map;
    };
    std::unique_ptr<TransShard[]> trans_;
    std::unordered_map<uint64_t, double> calib_;                // phase hash -> ns per work unit
    std::unordered_map<uint64_t, bool> mustWalk_;               // phase hash -> walk next time
    double defaultCalib_ = 1.0;
    std::atomic<size_t> cacheBytes_{0};
    // guards deg_ while the estimates of a build run on several threads
    // (entries are never erased during a build, so references handed out
    // stay valid)
    mutable std::shared_mutex cacheMu_;

    double sb_fan(int32_t pred, int dir);
    double avg_fan(const DevStep& st) const;
    double estimate(const PhasePlan& ph, bool hubAware);
    // Two-hop sums of the transition from (p0, d0) to (p1, d1), shared by
    // every plan whose first two steps follow it.
    const Hop2& hop2(int32_t p0, int d0, int32_t p1, int d1);
    // Plans whose second step is keyed by the value the first step binds.
    bool chain_shaped(const DevPlan& P) const;
    // Work per level-2 item: the product of the fan-outs of steps 2..m-1,
    // each through the step before it where the plan chains them.
    double chain_tail(const DevPlan& P);
    // Exact work of the first two levels times average fan-outs beyond, for
    // chain-shaped plans whose roots are the first step's rows; otherwise
    // the average-fan-out estimate.
    double estimate2(const PhasePlan& ph);
    const Walk& walk(const PhasePlan& ph, uint64_t sig);
    // The per-root walk of a phase (thread-safe: reads the index and the
    // lock-guarded estimate caches), and its insertion into the cache.
    Walk compute_walk(const PhasePlan& ph);
    const Walk& keep_walk(uint64_t sig, Walk&& wk);
    const Walk& walk(const PhasePlan& ph) { return walk(ph, phase_hash(ph)); }
    double child_work(const DevPlan& P, const int32_t* rootVals, int32_t e, const int32_t* deg2, double tail) const;

public:
    // Mean row length under (p1, d1) of the value an edge of (p0, d0) leads
    // to, over all edges of p0: the fan-out of a step reached through the
    // step before it (hub-heavy relations make it far above the plain
    // average).  capped: rows of kHubMinDegree edges or more count as
    // kHubMinDegree (a hub row of a body-size leaf is OR-ed a word at a time).
    // Cached; safe to call from several threads.
    double transition(int32_t p0, int d0, int32_t p1, int d1, bool capped);
    // The bound values of root r and the edge range of its first step: the
    // range a split root's slices [sub0, sub1) partition.
    int root_vals(const DevPlan& P, int32_t r, int32_t* vals) const;
    std::pair<int32_t, int32_t> first_segment(const DevPlan& P, int32_t r, const int32_t* vals) const;
};

}  // namespace gr
