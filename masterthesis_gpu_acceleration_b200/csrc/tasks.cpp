// tasks.cpp — balanced task construction (see tasks.hpp).
#include "tasks.hpp"
#include "parallel.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

namespace gr {
namespace {

constexpr double kMinTarget = 4096.0;
constexpr size_t kCacheLimit = size_t(2) << 30;

int64_t pd_key(int32_t pred, int dir) { return (int64_t)pred * 2 + dir; }


uint64_t signature(const PhasePlan& ph) { return phase_hash(ph); }

}  // namespace

namespace {
// The plan without its per-launch fields.
DevPlan plan_identity(const PhasePlan& ph) {
    DevPlan p = ph.plan;
    p.resultSlot = 0;
    p.gBitmap = nullptr;
    p.gRowBase = 0;
    p.gHeavy = nullptr;
    p.rowWords = 0;
    p.memoTab = nullptr;
    p.memoBits = nullptr;
    p.memoWords = 0;
    p.gBlockWords = 0;
    p.pairKeys = nullptr;
    p.keyCursor = nullptr;
    p.keyCap = 0;
    p.keyBase = 0;
    p.rankBits = 0;
    p.pad0 = 0;
    p.pad1 = 0;
    p.pad2 = 0;
    p.pad3 = 0;
    return p;
}
}  // namespace

bool phase_equal(const PhasePlan& a, const PhasePlan& b) {
    if (a.rootBeg != b.rootBeg || a.rootEnd != b.rootEnd) return false;
    const DevPlan pa = plan_identity(a), pb = plan_identity(b);
    return std::memcmp(&pa, &pb, sizeof(DevPlan)) == 0;
}

uint64_t phase_hash(const PhasePlan& ph) {
    static_assert(sizeof(DevPlan) % 8 == 0, "plan hashed in 8-byte words");
    const DevPlan p = plan_identity(ph);
    const unsigned char* b = reinterpret_cast<const unsigned char*>(&p);
    // four independent lanes (a quarter of the dependent multiplies each),
    // combined at the end
    uint64_t h[4] = {0x243F6A8885A308D3ull ^ ((uint64_t)(uint32_t)ph.rootBeg << 32 | (uint32_t)ph.rootEnd),
                     0x13198A2E03707344ull, 0xA4093822299F31D0ull, 0x082EFA98EC4E6C89ull};
    size_t i = 0;
    for (; i + 32 <= sizeof(DevPlan); i += 32)
        for (int k = 0; k < 4; ++k) {
            uint64_t w;
            std::memcpy(&w, b + i + 8 * k, 8);
            h[k] = (h[k] ^ w) * 0x9E3779B97F4A7C15ull;
            h[k] ^= h[k] >> 29;
        }
    for (int k = 0; i < sizeof(DevPlan); i += 8, ++k) {
        uint64_t w;
        std::memcpy(&w, b + i, 8);
        h[k] = (h[k] ^ w) * 0x9E3779B97F4A7C15ull;
        h[k] ^= h[k] >> 29;
    }
    uint64_t r = h[0];
    for (int k = 1; k < 4; ++k) {
        r = (r ^ h[k]) * 0xD6E8FEB86659FD93ull;
        r ^= r >> 32;
    }
    return r;
}

TaskBuilder::TaskBuilder(const HostIndex& ix)
    : ix_(ix), degAt_((size_t)std::max(ix.nPred, 0) * 2), sbFan_((size_t)std::max(ix.nPred, 0) * 2, 0.0),
      hop2_(new Hop2Shard[kHop2Shards]), trans_(new TransShard[kHop2Shards]) {
    for (auto& a : degAt_) a.store(nullptr, std::memory_order_relaxed);
    for (int32_t p = 0; p < ix.nPred; ++p)
        for (int dir = 0; dir < 2; ++dir) {
            double s1 = 0, s2 = 0;
            for (int32_t r = ix.predRow[dir][p]; r < ix.predRow[dir][p + 1]; ++r) {
                const double d = ix.rowBeg[dir][r + 1] - ix.rowBeg[dir][r];
                s1 += d;
                s2 += d * d;
            }
            sbFan_[(size_t)p * 2 + dir] = s1 > 0 ? s2 / s1 : 0.0;
        }
}

const int32_t* TaskBuilder::degrees(int32_t pred, int dir) {
    const size_t at = (size_t)pred * 2 + (size_t)dir;
    if (const int32_t* d = degAt_[at].load(std::memory_order_acquire)) return d;
    std::vector<int32_t> d((size_t)std::max(ix_.nEnt, 1), 0);
    for (int32_t r = ix_.predRow[dir][pred]; r < ix_.predRow[dir][pred + 1]; ++r)
        d[ix_.rowKey[dir][r]] = ix_.rowBeg[dir][r + 1] - ix_.rowBeg[dir][r];
    std::unique_lock<std::shared_mutex> lk(cacheMu_);
    auto ins = deg_.emplace(pd_key(pred, dir), std::move(d));
    if (ins.second) cacheBytes_ += ins.first->second.size() * 4;
    degAt_[at].store(ins.first->second.data(), std::memory_order_release);
    return ins.first->second.data();
}

double TaskBuilder::sb_fan(int32_t pred, int dir) { return sbFan_[(size_t)pred * 2 + (size_t)dir]; }

double TaskBuilder::avg_fan(const DevStep& st) const {
    if (st.kind == kScan) return (double)ix_.pred_size(st.pred);
    return std::max(1.0, ix_.avg_degree(st.pred, st.dir));
}

double TaskBuilder::estimate(const PhasePlan& ph, bool hubAware) {
    const DevPlan& P = ph.plan;
    double w = std::max(1, ph.rootEnd - ph.rootBeg);
    for (int s = 0; s < P.m; ++s) {
        const DevStep& st = P.steps[s];
        double f = avg_fan(st);
        if (hubAware && st.kind == kExpand) f = std::max(f, sb_fan(st.pred, st.dir));
        w *= std::max(1.0, f);
        if (w > 1e18) return 1e18;
    }
    return w;
}

const TaskBuilder::Hop2& TaskBuilder::hop2(int32_t p0, int d0, int32_t p1, int d1) {
    const uint64_t key = ((uint64_t)(uint32_t)p0 << 33) | ((uint64_t)d0 << 32) | ((uint64_t)(uint32_t)p1 << 1) | (uint64_t)d1;
    Hop2Shard& sh = hop2_[(key * 0x9E3779B97F4A7C15ull) >> 58];
    {
        std::shared_lock<std::shared_mutex> lk(sh.mu);
        auto it = sh.map.find(key);
        if (it != sh.map.end()) return it->second;
    }
    const int32_t* deg = degrees(p1, d1);
    Hop2 h;
    const int32_t r0 = ix_.predRow[d0][p0], r1 = ix_.predRow[d0][p0 + 1];
    h.perRow.resize((size_t)(r1 - r0));
    for (int32_t r = r0; r < r1; ++r) {
        double acc = 0;
        for (int32_t e = ix_.rowBeg[d0][r]; e < ix_.rowBeg[d0][r + 1]; ++e) acc += deg[ix_.val[d0][e]];
        h.perRow[r - r0] = (float)acc;
        h.total += acc;
    }
    std::unique_lock<std::shared_mutex> lk(sh.mu);
    auto ins = sh.map.emplace(key, std::move(h));
    if (ins.second) cacheBytes_ += ins.first->second.perRow.size() * sizeof(float);
    return ins.first->second;
}

double TaskBuilder::transition(int32_t p0, int d0, int32_t p1, int d1, bool capped) {
    const uint64_t key = ((uint64_t)(uint32_t)p0 << 34) | ((uint64_t)d0 << 33) | ((uint64_t)(uint32_t)p1 << 2) |
                         ((uint64_t)d1 << 1) | (capped ? 1u : 0u);
    TransShard& sh = trans_[(key * 0x9E3779B97F4A7C15ull) >> 58];
    {
        std::shared_lock<std::shared_mutex> lk(sh.mu);
        auto it = sh.map.find(key);
        if (it != sh.map.end()) return it->second;
    }
    // an edge of (p0, d0) leads to v as often as v's row under (p0, 1 - d0)
    // is long: one lookup per distinct v
    const int rd = 1 - d0;
    double n = 0, acc = 0;
    for (int32_t r = ix_.predRow[rd][p0]; r < ix_.predRow[rd][p0 + 1]; ++r) {
        const double c = ix_.rowBeg[rd][r + 1] - ix_.rowBeg[rd][r];
        const auto rr = ix_.row_range(p1, d1, ix_.rowKey[rd][r]);
        double d = rr.second - rr.first;
        if (capped) d = std::min(d, (double)kHubMinDegree);
        n += c;
        acc += c * d;
    }
    const double mean = n > 0 ? acc / n : 0.0;
    std::unique_lock<std::shared_mutex> lk(sh.mu);
    sh.map.emplace(key, mean);
    return mean;
}

double TaskBuilder::chain_tail(const DevPlan& P) {
    double tail = 1.0;
    for (int s = 2; s < P.m; ++s) {
        const DevStep& st = P.steps[s];
        const DevStep& pv = P.steps[s - 1];
        double f;
        if (st.kind == kExpand && pv.kind == kExpand && pv.nNew == 1 && st.keyRef == P.tupleLen[s - 1]) {
            const bool capped = s == P.m - 1 && P.mode == kPairs && P.hoLevel == P.m && !ix_.hubOff.empty();
            f = transition(pv.pred, pv.dir, st.pred, st.dir, capped);
        } else
            f = avg_fan(st);
        tail *= std::max(1.0, f);
    }
    return tail;
}

bool TaskBuilder::chain_shaped(const DevPlan& P) const {
    return P.m >= 2 && P.steps[0].kind == kExpand && P.steps[1].kind == kExpand &&
           P.steps[1].keyRef == P.tupleLen[0] && (P.steps[0].keyRef < 0 || P.steps[0].keyRef < P.tupleLen[0]);
}

double TaskBuilder::estimate2(const PhasePlan& ph) {
    const DevPlan& P = ph.plan;
    if (!chain_shaped(P)) return estimate(ph, false);
    const DevStep& s0 = P.steps[0];
    const DevStep& s1 = P.steps[1];
    // plain average fan-outs beyond the second step: this figure also sets
    // the serving loop's light/heavy lanes, whose latency measured better on
    // it (c3 + c4 at 5k requests/s: p99 394 ms against 917 ms with the
    // chained fan-outs that per-root walks use)
    double tail = 1.0;
    for (int s = 2; s < P.m; ++s) tail *= std::max(1.0, avg_fan(P.steps[s]));
    const Hop2& h = hop2(s0.pred, s0.dir, s1.pred, s1.dir);
    const bool allRows = P.rootKind == kRootRows && P.rootDir == s0.dir && P.rootPred == s0.pred &&
                         s0.keyRef == kTupleHead && ph.rootBeg == ix_.predRow[s0.dir][s0.pred] &&
                         ph.rootEnd == ix_.predRow[s0.dir][s0.pred + 1];
    if (allRows)
        return (double)(ph.rootEnd - ph.rootBeg) + (double)ix_.pred_size(s0.pred) + h.total * tail;
    // other roots: average first fan-out, and the transition's exact mean
    // second degree per first-level edge
    const double e0 = (double)std::max<int64_t>(1, ix_.pred_size(s0.pred));
    const double fan0 = std::max(1.0, ix_.avg_degree(s0.pred, s0.dir));
    return (double)(ph.rootEnd - ph.rootBeg) * (1.0 + fan0 * (1.0 + (h.total / e0) * tail));
}

int TaskBuilder::root_vals(const DevPlan& P, int32_t r, int32_t* vals) const {
    int nv = 0;
    if (P.rootKind == kRootRows) {
        vals[nv++] = ix_.rowKey[P.rootDir][r];
    } else {
        if (P.rootAppendKey) vals[nv++] = ix_.src[P.rootDir][r];
        if (P.rootAppendVal) vals[nv++] = ix_.val[P.rootDir][r];
    }
    return nv;
}

static int32_t resolve(const DevPlan& P, TermRef ref, const int32_t* vals, int32_t n0, int32_t n1) {
    if (ref < 0) return P.consts[-1 - ref];
    if (ref < kTupleHead) return -1;
    if (ref < P.tupleLen[0]) return vals[ref - kTupleHead];
    return ref == P.tupleLen[0] ? n0 : n1;
}

std::pair<int32_t, int32_t> TaskBuilder::first_segment(const DevPlan& P, int32_t r, const int32_t* vals) const {
    const DevStep& st = P.steps[0];
    if (st.kind == kScan) return {ix_.predEdge[0][st.pred], ix_.predEdge[0][st.pred + 1]};
    // the first step expands the root's own row: no lookup
    if (P.rootKind == kRootRows && P.rootDir == st.dir && P.rootPred == st.pred && st.keyRef == kTupleHead)
        return {ix_.rowBeg[st.dir][r], ix_.rowBeg[st.dir][r + 1]};
    return ix_.row_range(st.pred, st.dir, resolve(P, st.keyRef, vals, -1, -1));
}

double TaskBuilder::child_work(const DevPlan& P, const int32_t* vals, int32_t e, const int32_t* deg2,
                               double tail) const {
    if (P.m < 2) return 1.0;
    const DevStep& s0 = P.steps[0];
    int32_t n0, n1 = -1;
    if (s0.kind == kExpand) n0 = ix_.val[s0.dir][e];
    else { n0 = ix_.src[0][e]; n1 = ix_.val[0][e]; }
    const DevStep& s1 = P.steps[1];
    double d2;
    if (s1.kind == kScan) d2 = (double)ix_.pred_size(s1.pred);
    else {
        int32_t k = resolve(P, s1.keyRef, vals, n0, n1);
        d2 = (k >= 0 && k < ix_.nEnt) ? deg2[k] : 0.0;
    }
    return 1.0 + d2 * tail;
}

const TaskBuilder::Walk& TaskBuilder::walk(const PhasePlan& ph, uint64_t sig) {
    auto it = walks_.find(sig);
    if (it != walks_.end()) return it->second;
    return keep_walk(sig, compute_walk(ph));
}

const TaskBuilder::Walk& TaskBuilder::keep_walk(uint64_t sig, Walk&& wk) {
    cacheBytes_ += wk.w.size() * sizeof(float) + wk.bsum.size() * (sizeof(double) + sizeof(float)) + sizeof(Walk);
    return walks_.emplace(sig, std::move(wk)).first->second;
}

TaskBuilder::Walk TaskBuilder::compute_walk(const PhasePlan& ph) {
    const DevPlan& P = ph.plan;
    const double tail = chain_tail(P);
    const bool chain = chain_shaped(P);
    const Hop2* h = chain ? &hop2(P.steps[0].pred, P.steps[0].dir, P.steps[1].pred, P.steps[1].dir) : nullptr;
    const int32_t* deg2 = (!chain && P.m >= 2 && P.steps[1].kind == kExpand) ? degrees(P.steps[1].pred, P.steps[1].dir) : nullptr;
    // plans whose last two (three) steps are memoised: an item of level 1
    // costs the memo's price when its row has a memo, else its enumeration
    const std::vector<uint8_t>* memo = nullptr;
    double memoCost = 0.0;
    const DevStep& s1 = P.steps[1];
    if (chain && P.mode == kPairs && P.memoLevel == 2 && memoRows) {
        if (P.m == 3)
            memo = memoRows(s1.pred, s1.dir, P.steps[2].pred, P.steps[2].dir, -1, 0, &memoCost);
        else if (P.m == 4 && P.memoSteps == 3)
            memo = memoRows(s1.pred, s1.dir, P.steps[2].pred, P.steps[2].dir, P.steps[3].pred, P.steps[3].dir,
                            &memoCost);
    }
    // a second step that scans, or expands from a root value or a constant,
    // costs the same after every edge of the first step
    const bool uniformChild = P.m >= 2 && (s1.kind == kScan || s1.keyRef < P.tupleLen[0]);
    std::vector<float> w((size_t)(ph.rootEnd - ph.rootBeg));
    int32_t vals[2];
    for (int32_t r = ph.rootBeg; r < ph.rootEnd; ++r) {
        root_vals(P, r, vals);
        auto seg = first_segment(P, r, vals);
        double acc = 1.0;
        if (P.m < 2) acc += seg.second - seg.first;
        else if (chain && memo) {
            acc += seg.second - seg.first;
            const int d0 = P.steps[0].dir;
            for (int32_t e = seg.first; e < seg.second; ++e) {
                const auto rr = ix_.row_range(s1.pred, s1.dir, ix_.val[d0][e]);
                if (rr.second <= rr.first) continue;
                const int32_t row = ix_.srcRank[s1.dir][rr.first];   // row index within the predicate
                acc += (*memo)[(size_t)row] ? memoCost : (double)(rr.second - rr.first) * tail;
            }
        } else if (chain) {
            acc += seg.second - seg.first;
            if (seg.second > seg.first) acc += h->perRow[ix_.srcRank[P.steps[0].dir][seg.first]] * tail;
        } else if (uniformChild) {
            // the second step does not depend on the first step's value:
            // every edge of the segment costs the same
            if (seg.second > seg.first)
                acc += (double)(seg.second - seg.first) * child_work(P, vals, seg.first, deg2, tail);
        } else
            for (int32_t e = seg.first; e < seg.second; ++e) acc += child_work(P, vals, e, deg2, tail);
        w[r - ph.rootBeg] = (float)acc;
    }
    Walk entry;
    for (float x : w) entry.sum += x;
    const size_t nb = w.size() / kWalkBlock;
    entry.bsum.assign(nb, 0.0);
    entry.bmax.assign(nb, 0.f);
    for (size_t b = 0; b < nb; ++b)
        for (size_t k = b * kWalkBlock; k < (b + 1) * kWalkBlock; ++k) {
            entry.bsum[b] += w[k];
            entry.bmax[b] = std::max(entry.bmax[b], w[k]);
        }
    entry.w = std::move(w);
    return entry;
}

void TaskBuilder::build(const std::vector<const PhasePlan*>& phases, int blocks, bool split,
                        std::vector<PhaseTasks>& out, double walkBudget, bool costAware,
                        const std::vector<PhaseLimits>* limits) {
    size_t n = phases.size();
    out.assign(n, PhaseTasks{});
    if (cacheBytes_ > kCacheLimit) {  // only here: walks hand out references into the cache
        walks_.clear();
        deg_.clear();
        for (auto& a : degAt_) a.store(nullptr, std::memory_order_relaxed);
        for (int k = 0; k < kHop2Shards; ++k) {
            hop2_[k].map.clear();
            trans_[k].map.clear();
        }
        cacheBytes_ = 0;
    }
    std::vector<double> estAvg(n), estHub(n), scale(n, defaultCalib_);
    std::vector<const Walk*> walked(n, nullptr);
    std::vector<char> forced(n, 0);
    const bool learned = !calib_.empty() || !mustWalk_.empty();
    // signatures and cached-walk flags too: the walk cache only changes
    // after this loop
    std::vector<uint64_t> sig(n, 0);
    std::vector<char> cached(n, 0);
    parallel_for(n, [&](size_t i) {
        estAvg[i] = estimate2(*phases[i]);
        estHub[i] = split ? estimate(*phases[i], true) : estAvg[i];
        out[i].work = estAvg[i];
        if (learned || split) sig[i] = signature(*phases[i]);
        if (learned) {
            auto c = calib_.find(sig[i]);
            if (c != calib_.end()) scale[i] = c->second;
            forced[i] = mustWalk_.count(sig[i]) ? 1 : 0;
        }
        if (split) cached[i] = walks_.count(sig[i]) ? 1 : 0;
    }, 16);
    if (split) {
        std::vector<size_t> ord(n);
        std::iota(ord.begin(), ord.end(), 0);
        // phases that ran slow before come first, then the hub-aware ranking
        std::sort(ord.begin(), ord.end(), [&](size_t a, size_t b) {
            if (forced[a] != forced[b]) return forced[a] > forced[b];
            return estHub[a] > estHub[b];
        });
        double used = 0;
        std::vector<size_t> sel;          // phases that get a walk
        for (size_t i : ord) {
            if (!forced[i] && estHub[i] < walkThreshold) break;
            const PhasePlan& ph = *phases[i];
            const DevStep& s0 = ph.plan.steps[0];
            // cost of a walk: one lookup per root for chain-shaped plans,
            // otherwise every first-segment edge
            double edges = chain_shaped(ph.plan) ? (double)(ph.rootEnd - ph.rootBeg)
                         : (double)(ph.rootEnd - ph.rootBeg) *
                           (s0.kind == kExpand ? std::max(1.0, ix_.avg_degree(s0.pred, s0.dir)) : (double)ix_.pred_size(s0.pred));
            if (!forced[i] && !cached[i] && used + edges > walkBudget) continue;
            // a walk whose own cost exceeds the phase's expected device time
            // cannot pay for itself (a single rule on the whole GPU)
            if (costAware && !cached[i] && std::max(estAvg[i], estHub[i]) * scale[i] < kWalkNsPerEdge * edges) continue;
            if (!cached[i]) used += edges;   // cached walks cost nothing
            sel.push_back(i);
        }
        // the new walks, one per distinct signature, on host threads (a walk
        // only reads the index and the shared estimate caches)
        std::vector<size_t> fresh;
        {
            std::unordered_map<uint64_t, char> pending;
            for (size_t i : sel)
                if (!walks_.count(sig[i]) && pending.emplace(sig[i], 1).second) fresh.push_back(i);
        }
        std::vector<Walk> made(fresh.size());
        // threads only pay for themselves on large walks (~0.1 ms and up)
        parallel_for(fresh.size(), [&](size_t k) { made[k] = compute_walk(*phases[fresh[k]]); },
                     used > 1.0e5 ? 1 : fresh.size() + 1);
        for (size_t k = 0; k < fresh.size(); ++k) keep_walk(sig[fresh[k]], std::move(made[k]));
        for (size_t i : sel) {
            const Walk& wk = walks_.find(sig[i])->second;
            walked[i] = &wk;
            out[i].work = wk.sum;
        }
    }
    // work in device-time units (learned ns per unit, where known)
    double total = 0;
    for (size_t i = 0; i < n; ++i) total += out[i].work * scale[i];
    const double target = forceTarget > 0 ? forceTarget
                                          : std::max(kMinTarget * defaultCalib_, total / (std::max(blocks, 1) * 8.0));

    // task lists per phase: independent once the degree arrays that heavy
    // roots split by exist, so built in parallel
    for (size_t i = 0; i < n; ++i) {
        const DevPlan& P = phases[i]->plan;
        if (walked[i] && P.m >= 2 && P.steps[1].kind == kExpand) degrees(P.steps[1].pred, P.steps[1].dir);
    }
    parallel_for(n, [&](size_t i) {
        const PhasePlan& ph = *phases[i];
        const DevPlan& P = ph.plan;
        PhaseTasks& pt = out[i];
        const double sc = forceTarget > 0 ? 1.0 : scale[i];
        pt.scale = scale[i];
        int32_t g = std::max(P.groupMax, 1);
        if (ph.needsGlobalBitmap) g = std::min(P.cap, 512);
        const PhaseLimits lim = limits ? (*limits)[i] : PhaseLimits{};
        if (lim.group > 0) g = std::min(g, lim.group);
        const int32_t R = ph.rootEnd - ph.rootBeg;
        const double uniform = R > 0 ? std::max(1.0, pt.work / R) : 1.0;
        const Walk* wk = walked[i];
        if (!wk) {
            // uniform cost per root: fixed-size chunks, no per-root pass
            const double per = uniform * sc;
            int32_t chunk = g;
            if (per > 0 && per * chunk > target) chunk = std::max<int32_t>(1, (int32_t)(target / per));
            for (int32_t b = ph.rootBeg; b < ph.rootEnd; b += chunk) {
                const int32_t e = std::min(ph.rootEnd, b + chunk);
                pt.tasks.push_back(DevTask{(int32_t)i, b, e, 0, 0, -1});
                pt.cost.push_back(uniform * (e - b));
            }
            return;
        }
        int32_t gb = ph.rootBeg;
        double acc = 0, accUnits = 0;
        auto flush = [&](int32_t end) {
            if (end > gb) {
                pt.tasks.push_back(DevTask{(int32_t)i, gb, end, 0, 0, -1});
                pt.cost.push_back(accUnits);
            }
            gb = end;
            acc = 0;
            accUnits = 0;
        };
        const std::vector<float>& w = wk->w;
        const bool canSplit = split && P.m >= 1;
        // Roots heavier than splitAt are cut into slices of `target`.  A
        // launch of one rule (costAware) cuts only roots above a block's fair
        // share of the phase: lighter ones cannot hold up its end, and each
        // cut costs host time per first-segment edge.
        const double splitAt = costAware ? std::max(target, pt.work * sc / std::max(blocks, 1)) : target;
        const double tail = chain_tail(P);
        const int32_t* deg2 =
            (canSplit && P.m >= 2 && P.steps[1].kind == kExpand) ? degrees(P.steps[1].pred, P.steps[1].dir) : nullptr;
        for (int32_t r = ph.rootBeg; r < ph.rootEnd; ++r) {
            const int32_t o = r - ph.rootBeg;
            if (o % kWalkBlock == 0 && (size_t)(o / kWalkBlock) < wk->bsum.size()) {
                // a whole block that neither holds a heavy root nor ends the
                // current task (roots below exceed neither bound one by one)
                const size_t b = (size_t)(o / kWalkBlock);
                const double bs = wk->bsum[b];
                if ((!canSplit || (double)wk->bmax[b] * sc <= splitAt) && acc + bs * sc <= target &&
                    r + kWalkBlock - 1 - gb < g) {
                    acc += bs * sc;
                    accUnits += bs;
                    r += kWalkBlock - 1;
                    continue;
                }
            }
            const double wu = (double)w[o];
            const double wr = wu * sc;
            if (canSplit && wr > splitAt && (lim.maxHeavy < 0 || pt.heavyRows < lim.maxHeavy)) {
                // a heavy root: slices of its first segment, one task each
                flush(r);
                int32_t vals[2];
                root_vals(P, r, vals);
                auto seg = first_segment(P, r, vals);
                size_t first = pt.tasks.size();
                int32_t s0 = 0;
                double sa = 0;
                for (int32_t e = seg.first; e < seg.second; ++e) {
                    sa += child_work(P, vals, e, deg2, tail);
                    if (sa * sc >= target || e + 1 == seg.second) {
                        int32_t s1 = e + 1 - seg.first;
                        pt.tasks.push_back(DevTask{(int32_t)i, r, r + 1, s0, s1, pt.heavyRows});
                        pt.cost.push_back(sa);
                        s0 = s1;
                        sa = 0;
                    }
                }
                if (pt.tasks.size() - first <= 1) {
                    // not worth a global row: keep the root as a plain task
                    if (pt.tasks.size() > first) { pt.tasks.pop_back(); pt.cost.pop_back(); }
                    pt.tasks.push_back(DevTask{(int32_t)i, r, r + 1, 0, 0, -1});
                    pt.cost.push_back(wu);
                } else {
                    pt.heavyRows++;
                }
                gb = r + 1;
                continue;
            }
            if (r > gb && (r - gb >= g || acc + wr > target)) flush(r);
            acc += wr;
            accUnits += wu;
        }
        flush(ph.rootEnd);
    }, 8);
}

std::vector<int32_t> TaskBuilder::split_roots(const PhasePlan& ph, int n) {
    n = std::max(n, 1);
    std::vector<int32_t> cut(n + 1, ph.rootEnd);
    cut[0] = ph.rootBeg;
    const int32_t R = ph.rootEnd - ph.rootBeg;
    if (R <= 0) return cut;
    const std::vector<float>& w = walk(ph).w;
    double total = 0;
    for (float x : w) total += x;
    double acc = 0;
    int k = 1;
    for (int32_t r = 0; r < R && k < n; ++r) {
        acc += w[r];
        while (k < n && acc >= total * k / n) cut[k++] = ph.rootBeg + r + 1;
    }
    return cut;
}

double TaskBuilder::expected_ns(const PhasePlan& ph) {
    if (ph.how != kDevice) return 0.0;
    if (!calib_.empty()) {
        auto it = calib_.find(signature(ph));
        if (it != calib_.end()) return estimate2(ph) * it->second;
    }
    // the average-fan-out estimate, raised at most tenfold toward the
    // hub-aware one (which assumes every step lands on a hub)
    return estimate2(ph) * defaultCalib_;
}

void TaskBuilder::learn(const std::vector<const PhasePlan*>& phases, const std::vector<DevTask>& tasks,
                        const std::vector<double>& cost, const unsigned long long* taskNs, int blocks,
                        double weight, double minWorstNs) {
    size_t n = phases.size();
    std::vector<double> ns(n, 0.0), units(n, 0.0), worst(n, 0.0);
    double totNs = 0, totUnits = 0;
    for (size_t t = 0; t < tasks.size(); ++t) {
        int p = tasks[t].plan;
        if (p < 0 || (size_t)p >= n) continue;
        double d = (double)(taskNs[2 * t + 1] - taskNs[2 * t]);
        ns[p] += d;
        units[p] += std::max(cost[t], 1.0);
        worst[p] = std::max(worst[p], d);
        totNs += d;
        totUnits += std::max(cost[t], 1.0);
    }
    auto blend = [weight](double old, double now) { return old + weight * (now - old); };
    if (totUnits > 0) defaultCalib_ = blend(defaultCalib_, totNs / totUnits);
    const double limit = std::max(minWorstNs, totNs / (std::max(blocks, 1) * 8.0));
    for (size_t p = 0; p < n; ++p) {
        if (units[p] <= 0) continue;
        const uint64_t sig = signature(*phases[p]);
        auto it = calib_.find(sig);
        const double now = ns[p] / units[p];
        calib_[sig] = it == calib_.end() ? now : blend(it->second, now);
        if (worst[p] > limit) mustWalk_[sig] = true;
    }
}

}  // namespace gr
