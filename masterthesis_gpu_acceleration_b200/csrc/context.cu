// context.cu — graph context, staged launches and the C ABI
// (include/gpu_rules_api.h).
//
// Replaces the reference's GpuContext and entry points
// (GPU_03/gpu_rules_lib.cu:181-574).  Differences that matter to callers:
//  * errors are returned, never exit() (the reference's CUDA_OK calls exit,
//    GPU_03/gpu_common.cuh:8-15);
//  * unknown predicates and constants are resolved without growing the
//    dictionary (they match nothing, as a freshly interned id does);
//  * the body size is always computed (CPU_01 semantics), also when the
//    support is 0.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <chrono>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "engine.hpp"
#include "index_io.hpp"
#include "parallel.hpp"

namespace gr {

namespace {
thread_local std::string g_lastError;
}  // namespace

void set_error(const std::string& s) {
    g_lastError = s;
    std::fprintf(stderr, "[gpu_rules] %s\n", s.c_str());
}

namespace {
double host_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Plans whose leaf hub items may skip repeats (see kHubSeen): the leaf
// tuple holds hS and two more values, the leaf step expands from one of
// those two, binds hO and tests nothing but injectivity.
bool hub_leaf_claims(const DevPlan& P) {
    if (P.mode != kPairs || P.m < 1) return false;
    const DevStep& st = P.steps[P.m - 1];
    return P.tupleLen[P.m - 1] == kTupleHead + 3 && st.kind == kExpand && st.nNew == 1 && st.hoWhich != 0 &&
           (st.keyRef == kTupleHead + 1 || st.keyRef == kTupleHead + 2) && P.chkN[P.m] == 0 && P.usedN[P.m] == 0;
}

// Bits that hold the values 0 .. n - 1 (at least one).
int bits_for(uint64_t n) {
    int b = 1;
    while (b < 64 && n > 1 && ((n - 1) >> b) != 0) ++b;
    return b;
}
constexpr unsigned long long kMaxSortKeys = 0xffffffffull;   // the sort's 32-bit positions
}  // namespace

void Staged::stage(Context& c, std::vector<DevPlan>& plans, const std::vector<const PhasePlan*>& phases,
                   bool sortTasks, cudaStream_t s, double walkBudget, bool costAware, bool allowSort) {
    nPlans = (int)plans.size();
    nResults = nPlans + extraResults;
    stagedBlock = c.geom.block;
    nTasks = 0;
    bitmapWords = 0;
    blockWords = blockRegions = 0;
    nSort = sortBits = sortSlotShift = 0;
    keyCap = 0;
    h2dBytes = d2hBytes = 0;
    dedup.assign(nPlans, kDedupShared);
    const unsigned long long hint = keyHint;   // consumed by this staging
    keyHint = 0;
    if (hint > kMaxSortKeys) allowSort = false;
    if (!nPlans) return;

    double tSect = host_ms();
    // ---- how each kPairs plan deduplicates ----
    // Per-phase global rows (one bitmap row per root, cleared before the
    // launch) while all of them fit the budget.  Beyond it, per plan: sort
    // mode when the estimated keys (sorted in ~7 passes of 8 bits) cost fewer
    // bytes than clearing and setting the rows, else block rows, whose
    // memory grows with the launch's blocks instead of the phase's roots.
    const size_t budgetWords = std::max<size_t>(c.dedupBudget / 4, 1);
    std::vector<size_t> fullWords(nPlans, 0);
    std::vector<double> est(nPlans, -1.0);
    auto estimate = [&](int i) {
        if (est[i] < 0) est[i] = std::max(1.0, c.tasks->work_estimate(*phases[i]));
        return est[i];
    };
    size_t fullTotal = 0;
    for (int i = 0; i < nPlans; ++i) {
        if (plans[i].mode != kPairs || (!phases[i]->needsGlobalBitmap && c.dedupForce == 0)) continue;
        fullWords[i] = (size_t)(phases[i]->rootEnd - phases[i]->rootBeg) * (size_t)std::max(plans[i].rowWords, 1);
        fullTotal += fullWords[i];
        dedup[i] = kDedupRows;
    }
    for (int i = 0; i < nPlans; ++i) {
        if (dedup[i] == kDedupShared) continue;
        if (c.dedupForce) {
            dedup[i] = c.dedupForce;
        } else if (fullTotal > budgetWords) {
            const double e = estimate(i);
            const double rowBytes = 4.0 * (double)fullWords[i] + 8.0 * e;
            const double sortBytes = 8.0 * e * 22.0;
            dedup[i] = (sortBytes < rowBytes && 16.0 * e <= (double)c.dedupBudget) ? kDedupSort : kDedupBlockRows;
        }
        if (dedup[i] == kDedupSort && !allowSort) dedup[i] = kDedupBlockRows;
    }
    // sort keys: [sort index | row | rank], at most 64 bits
    std::vector<int32_t> sortPlans;
    int rankBits = 1, rowBits = 1;
    for (int i = 0; i < nPlans; ++i)
        if (dedup[i] == kDedupSort) {
            sortPlans.push_back(i);
            rankBits = std::max(rankBits, bits_for((uint64_t)std::max(plans[i].wo, 1)));
            rowBits = std::max(rowBits, bits_for((uint64_t)std::max(phases[i]->rootEnd - phases[i]->rootBeg, 1)));
        }
    if (!sortPlans.empty()) {
        const int slotBits = sortPlans.size() > 1 ? bits_for(sortPlans.size()) : 0;
        if (rankBits + rowBits + slotBits > 64) {
            for (int i : sortPlans) dedup[i] = kDedupBlockRows;
            sortPlans.clear();
        } else {
            nSort = (int)sortPlans.size();
            sortSlotShift = rankBits + rowBits;
            sortBits = sortSlotShift + slotBits;
        }
    }
    if (nSort) {
        // kept so that a run whose keys overflow can be staged again
        inPlans = plans;
        inPhases = phases;
        inSortTasks = sortTasks;
        inWalk = walkBudget;
        inCostAware = costAware;
        inAllowSort = allowSort;
    } else {
        inPlans.clear();
        inPhases.clear();
    }
    // block rows: every resident block owns a region that holds its current
    // task's rows; tasks are cut to the rows a region holds
    std::vector<PhaseLimits> lim(nPlans);
    {
        size_t maxRow = 0;
        for (int i = 0; i < nPlans; ++i)
            if (dedup[i] == kDedupBlockRows) maxRow = std::max(maxRow, (size_t)std::max(plans[i].rowWords, 1));
        if (maxRow) {
            blockRegions = (size_t)std::max(c.grid, 1);
            const size_t regionCap = std::max(maxRow, budgetWords / blockRegions);
            size_t need = 0;
            for (int i = 0; i < nPlans; ++i) {
                if (dedup[i] != kDedupBlockRows) continue;
                const size_t rw = (size_t)std::max(plans[i].rowWords, 1);
                const int32_t g = (int32_t)std::max<size_t>(
                    1, std::min<size_t>(regionCap / rw, (size_t)std::max(1, std::min(plans[i].cap, 512))));
                lim[i].group = g;
                lim[i].maxHeavy = (int32_t)std::min<size_t>(INT_MAX, budgetWords / 4 / rw);
                need = std::max(need, (size_t)g * rw);
            }
            blockWords = (need + 3) & ~size_t(3);
        }
    }
    std::vector<size_t> gOff(nPlans, 0);
    for (int i = 0; i < nPlans; ++i) {
        if (dedup[i] != kDedupRows) continue;
        gOff[i] = bitmapWords;
        bitmapWords += fullWords[i];   // word-aligned rows
    }
    const size_t regionOff = (bitmapWords + 3) & ~size_t(3);   // 16-byte aligned regions
    cudaStream_t as = streamOrdered ? s : nullptr;
    if (bitmapWords || blockWords) dBitmap.ensure((regionOff + blockRegions * blockWords) * 4, as);
    if (nSort) {
        double want = 0;
        for (int i : sortPlans) want += estimate(i);
        const double lo = 65536.0, hi = std::max(lo, (double)c.dedupBudget / 16.0);
        keyCap = (unsigned long long)std::min(hi, std::max(lo, want));
        keyCap = std::min(std::max(keyCap, hint), kMaxSortKeys);
        dSort.ensure(256 + (size_t)keyCap * 16 + pairs_sort_hist_words(keyCap) * 4, as);
        hSort.ensure(8);
    }
    hostSect[0] += host_ms() - tSect;
    tSect = host_ms();
    // suffix memos first: the task builder weighs memoised roots by them
    std::vector<std::array<int, 6>> memoKeys;
    auto memo_key_of = [](const DevPlan& P) -> std::array<int, 6> {
        const DevStep& a = P.steps[P.memoLevel - 1];
        if (P.memoSteps == 3) {
            const DevStep& c3 = P.steps[P.memoLevel + 1];
            return {a.pred, a.dir, P.memoP2, P.memoD2, c3.pred, c3.dir};
        }
        return {a.pred, a.dir, P.memoP2, P.memoD2, -1, 0};
    };
    for (int i = 0; i < nPlans; ++i) {
        if (plans[i].memoSteps == 3 && !c.memo3) {   // three-step memos switched off: enumerate
            plans[i].memoLevel = 0;
            plans[i].memoSteps = 0;
        }
        if (plans[i].memoLevel > 0 && dedup[i] != kDedupSort) memoKeys.push_back(memo_key_of(plans[i]));
    }
    if (!memoKeys.empty()) c.ensure_memos(memoKeys, s);
    hostSect[1] += host_ms() - tSect;
    tSect = host_ms();
    std::vector<PhaseTasks> pts;
    c.tasks->build(phases, c.grid, true, pts, walkBudget, costAware, &lim);
    hostSect[2] += host_ms() - tSect;
    tSect = host_ms();
    // split heavy roots of plans with fused support: counted after the launch
    std::vector<SupJob> supJobs;
    for (int i = 0; i < nPlans; ++i) {
        if (plans[i].supN == 0 || pts[i].heavyRows == 0) continue;
        std::vector<char> seenRow((size_t)pts[i].heavyRows, 0);
        for (const DevTask& t : pts[i].tasks)
            if (t.gRow >= 0 && !seenRow[(size_t)t.gRow]) {
                seenRow[(size_t)t.gRow] = 1;
                supJobs.push_back(SupJob{i, t.beg, t.gRow, 0});
            }
    }
    nSupJobs = (int)supJobs.size();
    std::vector<size_t> hOff(nPlans, 0);
    heavyWords = 0;
    for (int i = 0; i < nPlans; ++i) {
        plans[i].rowWords = plans[i].mode == kPairs ? (plans[i].wo + 31) / 32 : 1;
        hOff[i] = heavyWords;
        if (dedup[i] != kDedupSort) heavyWords += (size_t)pts[i].heavyRows * plans[i].rowWords;   // keys need no rows
    }
    if (heavyWords) dHeavy.ensure(heavyWords * 4, as);
    std::vector<DevTask> tasks;
    std::vector<double> cost;
    bool anyClaims = false;
    for (int i = 0; i < nPlans; ++i) anyClaims |= c.hubClaims && dedup[i] != kDedupSort && hub_leaf_claims(plans[i]);
    if (anyClaims) dHubSeen.ensure((size_t)std::max(c.grid, 1) * kHubSeen * 8, as);
    for (int i = 0; i < nPlans; ++i) {
        plans[i].memoTab = nullptr;
        plans[i].memoBits = nullptr;
        if (plans[i].memoLevel > 0) {
            const std::array<int, 6> k = memo_key_of(plans[i]);
            const SuffixMemo* m = c.memo_for(k[0], k[1], k[2], k[3], k[4], k[5]);
            if (m && (plans[i].mode != kPairs || m->words == plans[i].rowWords) &&
                (plans[i].memoSteps != 3 || m->wo == plans[i].wo)) {
                plans[i].memoTab = m->tab;
                plans[i].memoBits = m->bits;
                plans[i].memoWords = m->words;
            }
        }
        plans[i].resultSlot = i;
        const int dm = dedup[i];
        uint32_t* gb = static_cast<uint32_t*>(dBitmap.p);
        plans[i].gBitmap = dm == kDedupRows ? gb + gOff[i] : (dm == kDedupBlockRows ? gb + regionOff : nullptr);
        plans[i].gRowBase = (dm == kDedupRows || dm == kDedupSort) ? phases[i]->rootBeg : 0;
        plans[i].gBlockWords = dm == kDedupBlockRows ? (int64_t)blockWords : 0;
        plans[i].gHeavy = (pts[i].heavyRows && dm != kDedupSort) ? static_cast<uint32_t*>(dHeavy.p) + hOff[i] : nullptr;
        plans[i].hubSeen = (anyClaims && dm != kDedupSort && hub_leaf_claims(plans[i]))
                               ? static_cast<unsigned long long*>(dHubSeen.p) : nullptr;
        plans[i].pairKeys = nullptr;
        plans[i].keyCursor = nullptr;
        plans[i].keyCap = 0;
        plans[i].keyBase = 0;
        plans[i].rankBits = 0;
        if (dm == kDedupSort) {
            const int k = (int)(std::find(sortPlans.begin(), sortPlans.end(), i) - sortPlans.begin());
            char* sb = static_cast<char*>(dSort.p);
            plans[i].keyCursor = reinterpret_cast<unsigned long long*>(sb);
            plans[i].pairKeys = reinterpret_cast<unsigned long long*>(sb + 256);
            plans[i].keyCap = keyCap;
            plans[i].keyBase = (unsigned long long)k << sortSlotShift;
            plans[i].rankBits = rankBits;
            plans[i].memoTab = nullptr;   // memos set bitmap words; keys carry every pair
            plans[i].memoBits = nullptr;
        }
        tasks.insert(tasks.end(), pts[i].tasks.begin(), pts[i].tasks.end());
        cost.insert(cost.end(), pts[i].cost.begin(), pts[i].cost.end());
    }
    hostSect[3] += host_ms() - tSect;
    tSect = host_ms();
    if (sortTasks && tasks.size() > 1) {
        // longest (estimated device time) first, so the tail of the launch is
        // short: a stable counting sort by quarter-octaves of the estimate
        constexpr int kBuckets = 1024;
        auto bucket = [](double v) {
            if (!(v > 0.0)) return 0;
            int e;
            const double m = std::frexp(v, &e);   // v = m * 2^e, m in [0.5, 1)
            return std::max(1, std::min(kBuckets - 1, 512 + 4 * e + (int)((m - 0.5) * 8.0)));
        };
        std::vector<uint16_t> bk(tasks.size());
        std::vector<size_t> start(kBuckets + 1, 0);
        for (size_t i = 0; i < tasks.size(); ++i) {
            bk[i] = (uint16_t)bucket(cost[i] * pts[tasks[i].plan].scale);
            ++start[kBuckets - 1 - bk[i]];
        }
        size_t acc = 0;
        for (int b = 0; b <= kBuckets; ++b) { const size_t c = start[b]; start[b] = acc; acc += c; }
        std::vector<DevTask> t2(tasks.size());
        std::vector<double> c2(tasks.size());
        for (size_t i = 0; i < tasks.size(); ++i) {
            const size_t at = start[kBuckets - 1 - bk[i]]++;
            t2[at] = tasks[i];
            c2[at] = cost[i];
        }
        tasks.swap(t2);
        cost.swap(c2);
    }
    nTasks = (int)tasks.size();
    planTaskEnd.clear();
    if (!sortTasks) {
        // one launch per plan: each plan's tasks stay contiguous, longest
        // first within the plan
        int32_t acc = 0;
        std::vector<int32_t> ord;
        for (int i = 0; i < nPlans; ++i) {
            const int32_t b = acc, e = acc + (int32_t)pts[i].tasks.size();
            ord.resize((size_t)(e - b));
            std::iota(ord.begin(), ord.end(), b);
            std::stable_sort(ord.begin(), ord.end(), [&](int32_t x, int32_t y) { return cost[x] > cost[y]; });
            for (int32_t k = b; k < e; ++k) {
                pts[i].tasks[k - b] = tasks[ord[k - b]];
                pts[i].cost[k - b] = cost[ord[k - b]];
            }
            std::copy(pts[i].tasks.begin(), pts[i].tasks.end(), tasks.begin() + b);
            std::copy(pts[i].cost.begin(), pts[i].cost.end(), cost.begin() + b);
            planTaskEnd.push_back(acc = e);
        }
    }
    hostSect[4] += host_ms() - tSect;
    tSect = host_ms();
    size_t planBytes = (size_t)nPlans * sizeof(DevPlan);
    size_t taskBytes = (size_t)nTasks * sizeof(DevTask);
    const size_t sortBytes = ((size_t)nSort * sizeof(int32_t) + 15) & ~size_t(15);
    size_t blob = planBytes + taskBytes + sortBytes + (size_t)nSupJobs * sizeof(SupJob);
    hBlob.ensure(blob);
    std::memcpy(hBlob.p, plans.data(), planBytes);
    std::memcpy(static_cast<char*>(hBlob.p) + planBytes, tasks.data(), taskBytes);
    if (nSort) std::memcpy(static_cast<char*>(hBlob.p) + planBytes + taskBytes, sortPlans.data(), nSort * sizeof(int32_t));
    if (nSupJobs)
        std::memcpy(static_cast<char*>(hBlob.p) + planBytes + taskBytes + sortBytes, supJobs.data(),
                    (size_t)nSupJobs * sizeof(SupJob));
    hTasks = std::move(tasks);   // kept for profiles and task-time learning
    hCost = std::move(cost);
    dBlob.ensure(blob, as);
    nResults = nPlans + extraResults;
    dResults.ensure((size_t)nResults * sizeof(unsigned long long), as);
    dCtl.ensure(64, as);
    hResults.ensure((size_t)nResults * sizeof(unsigned long long));
    hCtl.ensure(64);
    ck(cudaMemcpyAsync(dBlob.p, hBlob.p, blob, cudaMemcpyHostToDevice, s), "H2D plans");
    dPlans = static_cast<const DevPlan*>(dBlob.p);
    dTasks = reinterpret_cast<const DevTask*>(static_cast<const char*>(dBlob.p) + planBytes);
    dSortSlots = nSort ? reinterpret_cast<const int32_t*>(static_cast<const char*>(dBlob.p) + planBytes + taskBytes)
                       : nullptr;
    dSupJobs = nSupJobs ? reinterpret_cast<const SupJob*>(static_cast<const char*>(dBlob.p) + planBytes + taskBytes +
                                                          sortBytes)
                        : nullptr;
    h2dBytes = blob;
    d2hBytes = (size_t)nResults * sizeof(unsigned long long) + 8;
    hostSect[5] += host_ms() - tSect;
}

namespace {
// Two-step memos keep the task builder's key ((p1, d1) and (p2, d2) in 32
// bits each); three-step keys set the top bit and pack 21 bits per step.
uint64_t memo_key(int p1, int d1, int p2, int d2, int p3 = -1, int d3 = 0) {
    if (p3 < 0) return ((uint64_t)(uint32_t)(p1 * 2 + d1) << 32) | (uint32_t)(p2 * 2 + d2);
    return (1ull << 63) | ((uint64_t)(uint32_t)(p1 * 2 + d1) << 42) | ((uint64_t)(uint32_t)(p2 * 2 + d2) << 21) |
           (uint64_t)(uint32_t)(p3 * 2 + d3);
}
}  // namespace

const SuffixMemo* Context::memo_for(int p1, int d1, int p2, int d2, int p3, int d3) const {
    auto it = memos.find(memo_key(p1, d1, p2, d2, p3, d3));
    return it == memos.end() ? nullptr : it->second.get();
}

void Context::ensure_memos(const std::vector<std::array<int, 6>>& keys, cudaStream_t s) {
    const HostIndex& h = hix;
    const int nHub = (int)h.hubOff.size();
    std::vector<std::array<int, 6>> fresh;
    for (const auto& k : keys) {
        const int p1 = k[0], p2 = k[2], p3 = k[4];
        const uint64_t key = memo_key(k[0], k[1], k[2], k[3], k[4], k[5]);
        if (memos.count(key)) continue;
        memos[key] = nullptr;
        if (memoGain < 0 || nHub == 0 || p1 < 0 || p2 < 0 || p1 >= h.nPred || p2 >= h.nPred || p3 >= h.nPred) continue;
        if (p3 >= 0 && h.nPred >= (1 << 20)) continue;
        fresh.push_back(k);
    }
    if (fresh.empty()) return;
    // the rank domain of a memo: the rows of its last step's predicate in
    // the other direction
    auto domain = [&](const std::array<int, 6>& k) -> int64_t {
        return k[4] >= 0 ? h.pred_rows(k[4], 1 - k[5]) : h.pred_rows(k[2], 1 - k[3]);
    };
    // the hub rows of (p1, d1) worth a memo, per new key, on host threads:
    // a row's candidates are what enumeration would visit from x on (its
    // own values, most of which may fail the next step's signature test,
    // and what they lead to)
    std::vector<std::vector<int32_t>> rowsOf(fresh.size());
    parallel_for(fresh.size(), [&](size_t i) {
        const int p1 = fresh[i][0], d1 = fresh[i][1], p2 = fresh[i][2], d2 = fresh[i][3];
        const int p3 = fresh[i][4], d3 = fresh[i][5];
        const int words = (int)((domain(fresh[i]) + 31) / 32);
        const double need = memoGain * words;
        // the count only grows: a row stops being summed once it qualifies
        // (a hub row's own values mostly do), and the degree array is made
        // only for a row that needs it
        const int32_t* deg = nullptr;
        for (int32_t r = h.predRow[d1][p1]; r < h.predRow[d1][p1 + 1]; ++r) {
            if (h.hubOf[d1][r] < 0) continue;
            double cand = (double)(h.rowBeg[d1][r + 1] - h.rowBeg[d1][r]);
            for (int32_t e = h.rowBeg[d1][r]; e < h.rowBeg[d1][r + 1] && cand < need; ++e) {
                if (!deg) deg = tasks->degrees(p3 >= 0 ? p3 : p2, p3 >= 0 ? d3 : d2);
                if (p3 < 0) {
                    cand += deg[h.val[d1][e]];
                } else {
                    const auto r2 = h.row_range(p2, d2, h.val[d1][e]);
                    for (int32_t e2 = r2.first; e2 < r2.second; ++e2) cand += 1.0 + deg[h.val[d2][e2]];
                }
            }
            if (cand >= need) rowsOf[i].push_back(r);
        }
    }, 1);
    // per memo slot: S1 and S2 (two steps), or S1 and one count per rank
    auto slot_words = [&](const std::array<int, 6>& k) -> size_t {
        const size_t words = (size_t)((domain(k) + 31) / 32);
        return k[4] >= 0 ? words + (size_t)(domain(k) + 3) / 4 : 2 * words;
    };
    // within the memory budget, in key order: one device allocation holding
    // every new memo's hub table, then every new memo's bits
    const size_t tabBytes = ((size_t)nHub * 4 + 255) & ~size_t(255);
    std::vector<size_t> take, bitOff;
    size_t bitTotal = 0;
    for (size_t i = 0; i < fresh.size(); ++i) {
        const size_t bytes = tabBytes + rowsOf[i].size() * slot_words(fresh[i]) * 4;
        if (rowsOf[i].empty() || memoBytes + bytes > kMemoBudgetBytes) continue;
        memoBytes += bytes;
        take.push_back(i);
        bitOff.push_back(bitTotal);
        bitTotal += rowsOf[i].size() * slot_words(fresh[i]) * 4;
    }
    if (take.empty()) return;
    const size_t tabTotal = tabBytes * take.size();
    memoChunks.emplace_back(new DevBuf());
    DevBuf& chunk = *memoChunks.back();
    ck(cudaMalloc(&chunk.p, tabTotal + bitTotal), "cudaMalloc(memos)");   // exact: never resized
    chunk.cap = tabTotal + bitTotal;
    char* base = static_cast<char*>(chunk.p);
    std::vector<int32_t> tabs(tabTotal / 4, -1);
    std::vector<MemoJob> all;
    for (size_t t = 0; t < take.size(); ++t) {
        const size_t i = take[t];
        const int p1 = fresh[i][0], d1 = fresh[i][1], p2 = fresh[i][2], d2 = fresh[i][3];
        const int p3 = fresh[i][4], d3 = fresh[i][5];
        const int wo = (int)domain(fresh[i]);
        const int words = (wo + 31) / 32;
        const size_t stride = slot_words(fresh[i]);
        int32_t* tab = tabs.data() + t * (tabBytes / 4);
        uint32_t* bits = reinterpret_cast<uint32_t*>(base + tabTotal + bitOff[t]);
        auto m = std::make_unique<SuffixMemo>();
        m->rowHasMemo.assign((size_t)h.pred_rows(p1, d1), 0);
        const std::vector<int32_t>& rows = rowsOf[i];
        for (size_t j = 0; j < rows.size(); ++j) {
            tab[h.hubOf[d1][rows[j]]] = (int32_t)j;
            m->rowHasMemo[(size_t)(rows[j] - h.predRow[d1][p1])] = 1;
            if (p3 < 0) {
                all.push_back(MemoJob{p1, d1, p2, d2, rows[j], words, p3, d3, wo, 0, -1, 0, bits + j * stride});
                continue;
            }
            // three steps: one block per slice of the row's values, so that
            // the paths of a long row spread over the SMs
            constexpr int32_t kSlice = 64;
            const int32_t len = h.rowBeg[d1][rows[j] + 1] - h.rowBeg[d1][rows[j]];
            for (int32_t b0 = 0; b0 < len; b0 += kSlice)
                all.push_back(MemoJob{p1, d1, p2, d2, rows[j], words, p3, d3, wo, b0, std::min(len, b0 + kSlice), 0,
                                      bits + j * stride});
        }
        m->tab = reinterpret_cast<const int32_t*>(base + t * tabBytes);
        m->bits = bits;
        m->words = words;
        m->wo = p3 >= 0 ? wo : 0;
        m->slots = (int)rows.size();
        memos[memo_key(p1, d1, p2, d2, p3, d3)] = std::move(m);
    }
    ck(cudaMemcpyAsync(base, tabs.data(), tabTotal, cudaMemcpyHostToDevice, s), "H2D memo tables");
    ck(cudaMemsetAsync(base + tabTotal, 0, bitTotal, s), "clear memo bits");
    memoJobs.ensure(all.size() * sizeof(MemoJob));
    ck(cudaMemcpyAsync(memoJobs.p, all.data(), all.size() * sizeof(MemoJob), cudaMemcpyHostToDevice, s),
       "H2D memo jobs");
    int maxWo = 0;
    for (const MemoJob& j : all)
        if (j.p3 >= 0) maxWo = std::max(maxWo, j.wo);
    ck(memo_build(dix, static_cast<const MemoJob*>(memoJobs.p), (int)all.size(), maxWo, s), "memo build");
    ck(cudaStreamSynchronize(s), "memo build");   // memos are shared by every stream afterwards
}

void Staged::enqueue_sort(Context& c, cudaStream_t s, unsigned long long* results, int* status) {
    if (!nSort) return;
    char* base = static_cast<char*>(dSort.p);
    auto* cursor = reinterpret_cast<unsigned long long*>(base);
    auto* keys = reinterpret_cast<unsigned long long*>(base + 256);
    auto* tmp = keys + keyCap;
    auto* hist = reinterpret_cast<uint32_t*>(tmp + keyCap);
    ck(pairs_sort_count(keys, tmp, cursor, keyCap, sortBits, sortSlotShift, dSortSlots, nSort, results, status,
                        hist, std::max(c.sms, 1) * 8, s),
       "pair sort");
}

void Staged::restage(Context& c, cudaStream_t s) {
    if (!nSort) return;
    keyHint = *static_cast<const unsigned long long*>(hSort.p);
    std::vector<DevPlan> p = inPlans;
    std::vector<const PhasePlan*> ph = inPhases;
    stage(c, p, ph, inSortTasks, s, inWalk, inCostAware, inAllowSort);
}

void Staged::check_geometry(const Context& c) const {
    // plans are laid out for the shared pool of the block size they were
    // staged at; a larger block's pool starts with it, a smaller one's is
    // too short (and its larger grid would outrun the per-block tables)
    if (c.geom.block < stagedBlock)
        throw CudaError("the launch's block size (" + std::to_string(c.geom.block) +
                        " threads) is below the one the plans were staged for (" + std::to_string(stagedBlock) +
                        "); prepare the batch again after changing the block size");
}

void Staged::enqueue(Context& c, cudaStream_t s, int instr, int gridCap, unsigned long long budgetNs) {
    budgeted = false;
    if (!nPlans) return;
    check_geometry(c);
    ck(cudaMemsetAsync(dResults.p, 0, (size_t)nResults * sizeof(unsigned long long), s), "memset results");
    ck(cudaMemsetAsync(dCtl.p, 0, 8, s), "memset ctl");
    if (bitmapWords) ck(cudaMemsetAsync(dBitmap.p, 0, bitmapWords * 4, s), "memset bitmap");
    if (heavyWords) ck(cudaMemsetAsync(dHeavy.p, 0, heavyWords * 4, s), "memset heavy rows");
    if (nSort) ck(cudaMemsetAsync(dSort.p, 0, 8, s), "memset key cursor");
    EngineProfile prof;
    if (instr >= 1) {
        dTaskNs.ensure((size_t)std::max(nTasks, 1) * 16, streamOrdered ? s : nullptr);
        prof.taskNs = static_cast<unsigned long long*>(dTaskNs.p);
    }
    if (instr >= 2) {
        dBytes.ensure(8, streamOrdered ? s : nullptr);
        ck(cudaMemsetAsync(dBytes.p, 0, 8, s), "memset bytes");
        prof.bytes = static_cast<unsigned long long*>(dBytes.p);
    }
    if (budgetNs && instr == 1) {
        dIncomplete.ensure((size_t)nPlans * sizeof(int), streamOrdered ? s : nullptr);
        hIncomplete.ensure((size_t)nPlans * sizeof(int));
        ck(cudaMemsetAsync(dIncomplete.p, 0, (size_t)nPlans * sizeof(int), s), "memset incomplete plans");
        prof.budgetNs = budgetNs;
        prof.incomplete = static_cast<int*>(dIncomplete.p);
        budgeted = true;
    }
    int grid = std::max(1, std::min(nTasks, gridCap > 0 ? std::min(gridCap, c.grid) : c.grid));
    if (blockWords && (size_t)grid > blockRegions) throw CudaError("launch grid exceeds the block-row regions");
    ck(engine_launch(c.dix, dPlans, dTasks, nTasks, static_cast<int*>(dCtl.p),
                     static_cast<unsigned long long*>(dResults.p), static_cast<int*>(dCtl.p) + 1, grid,
                     c.geom.block, s, instr ? &prof : nullptr),
       "engine launch");
    ck(support_rows(c.dix, dPlans, dSupJobs, nSupJobs, static_cast<unsigned long long*>(dResults.p), s),
       "fused support of split roots");
    enqueue_sort(c, s, static_cast<unsigned long long*>(dResults.p), static_cast<int*>(dCtl.p) + 1);
}

void Staged::enqueue_per_plan(Context& c, cudaStream_t s) {
    if (!nPlans) return;
    check_geometry(c);
    if (nPlans > kMaxPerPlan || (int)planTaskEnd.size() != nPlans) throw CudaError("bad per-plan staging");
    // control words: [0..1] task counters, [2] status (int), per plan two
    // u64 span words at byte 16 + 16 * i and its u64 result at
    // kPerPlanResults + 8 * i; all start at zero
    ck(cudaMemsetAsync(dCtl.p, 0, 64, s), "memset ctl");
    if (bitmapWords) ck(cudaMemsetAsync(dBitmap.p, 0, bitmapWords * 4, s), "memset bitmap");
    if (heavyWords) ck(cudaMemsetAsync(dHeavy.p, 0, heavyWords * 4, s), "memset heavy rows");
    if (nSort) ck(cudaMemsetAsync(dSort.p, 0, 8, s), "memset key cursor");
    int* ctl = static_cast<int*>(dCtl.p);
    for (int i = 0; i < nPlans; ++i) {
        const int32_t b = i ? planTaskEnd[i - 1] : 0, e = planTaskEnd[i];
        EngineProfile prof;
        prof.span = reinterpret_cast<unsigned long long*>(static_cast<char*>(dCtl.p) + 16 + 16 * i);
        const int grid = std::max(1, std::min(e - b, c.grid));
        if (blockWords && (size_t)grid > blockRegions) throw CudaError("launch grid exceeds the block-row regions");
        ck(engine_launch(c.dix, dPlans, dTasks + b, e - b, ctl + i,
                         reinterpret_cast<unsigned long long*>(static_cast<char*>(dCtl.p) + kPerPlanResults), ctl + 2,
                         grid, c.geom.block, s, &prof),
           "engine launch");
    }
    ck(support_rows(c.dix, dPlans, dSupJobs, nSupJobs,
                    reinterpret_cast<unsigned long long*>(static_cast<char*>(dCtl.p) + kPerPlanResults), s),
       "fused support of split roots");
    enqueue_sort(c, s, reinterpret_cast<unsigned long long*>(static_cast<char*>(dCtl.p) + kPerPlanResults), ctl + 2);
}

void Staged::download_spans(cudaStream_t s) {
    if (!nPlans) return;
    ck(cudaMemcpyAsync(hCtl.p, dCtl.p, 64, cudaMemcpyDeviceToHost, s), "D2H control words");
    download_cursor(s);
}

void compose(const RulePlan& rp, int64_t sup, int64_t body, double supMs, double confMs, GpuRuleResult* out) {
    *out = GpuRuleResult{};
    out->headSize = (int)clamp_int(rp.headSize);
    out->headSupport = (int)clamp_int(rp.headSupport);
    if (rp.status != kRuleOk) return;
    // FinalRule::setMeasures / setConfidence (CPU_01_nonparallel/FinalRule.cpp:19-41)
    int s = (int)clamp_int(sup), b = (int)clamp_int(body);
    out->support = s;
    out->headCoverage = out->headSize > 0 ? (double)s / (double)out->headSize : 0.0;
    out->bodySize = b;
    out->confidence = b > 0 ? (double)s / (double)b : 0.0;
    out->supportMs = supMs;
    out->confidenceMs = confMs;
}

namespace {

// One phase in its own launch (the plain per-rule form), timed by events.
int64_t run_one_phase(Context& c, const PhasePlan& ph, float* ms) {
    std::vector<DevPlan> plans{ph.plan};
    c.one.stage(c, plans, {&ph}, false, c.stream, c.ruleWalkBudget, true);
    for (int attempt = 0;; ++attempt) {
        ck(cudaEventRecord(c.ev[0], c.stream), "event");
        c.one.enqueue(c, c.stream, 0);
        ck(cudaEventRecord(c.ev[1], c.stream), "event");
        c.one.download(c.stream);
        ck(cudaStreamSynchronize(c.stream), "engine");
        c.one.check_status();
        if (attempt > 0 || !c.one.sort_overflow()) break;
        c.one.restage(c, c.stream);   // the exact key count is known now
    }
    ck(cudaEventElapsedTime(ms, c.ev[0], c.ev[1]), "elapsed");
    return (int64_t)c.one.counts()[0];
}

// Runs fn with the context's launch block size and grid switched to the
// per-rule block size, restoring them afterwards (also when fn throws).
// Only launches run under it: plans keep the batch geometry, whose shared
// pool is a prefix of the larger block's, so per-rule calls share the
// batch's cached walks and learnt costs (both keyed by plan signature).
template <class Fn>
void with_rule_block(Context& c, Fn fn) {
    struct Restore {
        Context& c;
        int block, grid;
        ~Restore() { c.geom.block = block; c.grid = grid; }
    } restore{c, c.geom.block, c.grid};
    if (c.ruleBlock > c.geom.block) c.set_block(c.ruleBlock);
    fn();
}

// Whether supports may be counted by their body-size plans (fused
// support, see RulePlan::supFuse): both phases run and no dedup mode is
// forced.
bool fusing(const Context& c) { return c.fuseSupport && (c.batchPhases & 3) == 3 && c.dedupForce == 0; }

// Both phases of one rule, each in its own launch timed by its own events,
// issued back to back with one host synchronisation; a fused support takes
// no launch of its own.
int evaluate_parsed(Context& c, const Rule& rule, GpuRuleResult* out) {
    RulePlan rp = plan_rule(rule, c.hix, c.geom);
    int64_t sup = rp.support.value, body = rp.body.value;
    float supMs = 0.f, confMs = 0.f;
    const bool runS = rp.status == kRuleOk && rp.support.how == kDevice;
    const bool runB = rp.status == kRuleOk && rp.body.how == kDevice;
    std::vector<DevPlan> plans;
    std::vector<const PhasePlan*> phases;
    // fused support (see prepare): the body-size launch also counts the
    // support, into per-plan result slot 1; the support takes no launch
    const bool fused = runS && runB && fusing(c) && rp.supFuse >= 0 && rp.body.plan.mode == kPairs &&
                       !rp.body.needsGlobalBitmap;
    if (runS && !fused) { plans.push_back(rp.support.plan); phases.push_back(&rp.support); }
    if (runB) { plans.push_back(rp.body.plan); phases.push_back(&rp.body); }
    if (fused) {
        DevPlan& B = plans.back();
        const auto dom = ho_domain(B);
        B.supN = 1;
        B.supDomPred = dom.first;
        B.supDomDir = dom.second;
        B.supPred[0] = rp.supFuse;
        B.supSlot[0] = 1;
    }
    if (!plans.empty()) {
        // one upload, one launch per phase (each timed on the device), one download
        c.one.stage(c, plans, phases, false, c.stream, c.ruleWalkBudget, true);
        for (int attempt = 0;; ++attempt) {
            with_rule_block(c, [&] { c.one.enqueue_per_plan(c, c.stream); });
            c.one.download_spans(c.stream);
            ck(cudaStreamSynchronize(c.stream), "engine");
            if (attempt > 0 || !c.one.sort_overflow()) break;
            c.one.restage(c, c.stream);   // the exact key count is known now
        }
        if (static_cast<const int*>(c.one.hCtl.p)[2] != 0)
            throw CudaError("engine reported internal status " + std::to_string(static_cast<const int*>(c.one.hCtl.p)[2]));
        int k = 0;
        if (runS && !fused) { sup = (int64_t)c.one.per_plan_count(k); supMs = (float)c.one.span_ms(k); ++k; }
        if (runB) { body = (int64_t)c.one.per_plan_count(k); confMs = (float)c.one.span_ms(k); }
        if (fused) sup = (int64_t)c.one.per_plan_count(1);   // counted by the body-size launch (supportMs 0)
    }
    compose(rp, sup, body, supMs, confMs, out);
    return 0;
}

// Counts of one rule restricted to slice `shard` of `nShards` of each device
// phase's roots (slices of about equal estimated work).  Support roots are
// head triples and body-size roots are rows of the seed atom keyed by the
// head subject, so the slices' counts add up to the whole rule's: distinct
// (hS, hO) pairs of different hS never collide.  Static parts count in
// slice 0 only.
void evaluate_shard(Context& c, const Rule& rule, int shard, int nShards, long long* counts) {
    RulePlan rp = plan_rule(rule, c.hix, c.geom);
    int64_t part[2] = {shard == 0 ? rp.support.value : 0, shard == 0 ? rp.body.value : 0};
    PhasePlan* phs[2] = {&rp.support, &rp.body};
    for (int k = 0; k < 2 && rp.status == kRuleOk; ++k) {
        PhasePlan& ph = *phs[k];
        if (ph.how != kDevice) continue;
        const std::vector<int32_t> cut = c.tasks->split_roots(ph, nShards);
        ph.rootBeg = cut[shard];
        ph.rootEnd = cut[shard + 1];
        part[k] = 0;
        float ms = 0.f;
        if (ph.rootEnd > ph.rootBeg) part[k] = run_one_phase(c, ph, &ms);
    }
    counts[0] = rp.status == kRuleOk ? part[0] : 0;
    counts[1] = rp.headSize;
    counts[2] = rp.headSupport;
    counts[3] = rp.status == kRuleOk ? part[1] : 0;
}

// Parses and plans n rules and stages their device phases.
// keepPlans: keep a copy of the plans for restaging (prepared batches that
// may be autotuned); one-shot chunks skip it.
void prepare(Batch& b, Context& c, const char* const* rules, int n, int isJson, bool keepPlans = true) {
    const double tStart = host_ms();
    b.c = &c;
    b.n = n;
    b.owner.clear();
    b.shared.clear();
    std::unordered_multimap<uint64_t, int> seen;
    seen.reserve(2 * (size_t)n);
    if (b.exec) { cudaGraphExecDestroy(b.exec); b.exec = nullptr; }
    if (b.graph) { cudaGraphDestroy(b.graph); b.graph = nullptr; }
    b.rps.assign(n, RulePlan{});
    b.parseStatus.assign(n, 0);
    std::vector<DevPlan> plans;
    std::vector<const PhasePlan*> phases;
    plans.reserve(2 * (size_t)n);
    std::vector<uint64_t> hash(2 * (size_t)n, 0);   // per rule: support and body phase hashes
    // parsing, planning and hashing only read the graph and the
    // dictionaries: in parallel
    parallel_for((size_t)n, [&](size_t i) {
        if (!rules[i]) { b.parseStatus[i] = -1; return; }
        try {
            Rule r = isJson ? c.parser->parse_json(rules[i]) : c.parser->parse_text(rules[i]);
            b.rps[i] = plan_rule(r, c.hix, c.geom);
            if (b.rps[i].status == kRuleOk) {
                if (b.rps[i].support.how == kDevice) hash[2 * i] = phase_hash(b.rps[i].support);
                if (b.rps[i].body.how == kDevice) hash[2 * i + 1] = phase_hash(b.rps[i].body);
            }
        } catch (const RuleError&) {
            b.parseStatus[i] = -1;
        }
    }, 16);
    // fused support: a rule whose support its body-size plan can count (see
    // RulePlan::supFuse) gets no support plan when that plan keeps its pair
    // rows in shared memory (no global dedup bitmap, no forced mode); the
    // count lands in a result slot after the plans' own
    const bool fuse = fusing(c);
    b.supOf.assign(n, -1);
    std::vector<std::array<int, 3>> fused;   // {body plan, head predicate, first rule}
    std::unordered_map<uint64_t, int> fusedAt;
    for (int i = 0; i < n; ++i) {
        if (b.parseStatus[i] != 0) continue;
        RulePlan& rp = b.rps[i];
        if (rp.status != kRuleOk) continue;
        int bodyPlan = -1;
        for (int k : {1, 0}) {
            const PhasePlan& ph = k == 0 ? rp.support : rp.body;
            if (ph.how != kDevice || !(c.batchPhases & (1 << k))) continue;
            if (k == 0 && fuse && rp.supFuse >= 0 && bodyPlan >= 0 && phases[bodyPlan]->plan.mode == kPairs &&
                !phases[bodyPlan]->needsGlobalBitmap) {
                const uint64_t key = ((uint64_t)(uint32_t)bodyPlan << 32) | (uint32_t)rp.supFuse;
                auto it = fusedAt.find(key);
                if (it != fusedAt.end()) {
                    b.supOf[i] = it->second;
                    continue;
                }
                DevPlan& B = plans[(size_t)bodyPlan];
                if (B.supN < kMaxSupFused) {
                    if (B.supN == 0) {
                        const auto dom = ho_domain(B);
                        B.supDomPred = dom.first;
                        B.supDomDir = dom.second;
                    }
                    B.supPred[B.supN] = rp.supFuse;
                    B.supSlot[B.supN] = (int32_t)fused.size();   // made absolute below
                    ++B.supN;
                    fusedAt.emplace(key, (int)fused.size());
                    b.supOf[i] = (int)fused.size();
                    fused.push_back({bodyPlan, rp.supFuse, i});
                    continue;
                }
            }
            // identical computations (same plan and roots, e.g. one body under
            // several heads) run once; the others share the count
            // keyed by hash, confirmed by the full signature (plans are
            // zero-initialised, so equal signatures mean equal computations)
            const uint64_t h = hash[2 * (size_t)i + k];
            auto range = seen.equal_range(h);
            int same = -1;
            for (auto it = range.first; it != range.second && same < 0; ++it)
                if (phase_equal(*phases[it->second], ph)) same = it->second;
            if (same >= 0) {
                b.shared.emplace_back(2 * i + k, same);
                if (k == 1) bodyPlan = same;
                continue;
            }
            seen.emplace(h, (int)plans.size());
            if (k == 1) bodyPlan = (int)plans.size();
            plans.push_back(ph.plan);
            phases.push_back(&ph);
            b.owner.push_back(2 * i + k);
        }
    }
    // fused counts follow the plans' own result slots
    const int nPlansOwn = (int)plans.size();
    for (DevPlan& P : plans)
        for (int j = 0; j < P.supN; ++j) P.supSlot[j] += nPlansOwn;
    for (int i = 0; i < n; ++i)
        if (b.supOf[i] >= 0) b.supOf[i] += nPlansOwn;
    b.st.extraResults = (int)fused.size();
    if (!b.stream) ck(cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking), "cudaStreamCreate");
    if (!b.ev0) ck(cudaEventCreate(&b.ev0), "cudaEventCreate");
    if (!b.ev1) ck(cudaEventCreate(&b.ev1), "cudaEventCreate");
    if (keepPlans) b.plans0 = plans;
    else b.plans0.clear();
    b.phases = phases;
    // a one-shot batch walks a phase only when the walk costs less host time
    // than the phase is expected to take on the device; a prepared batch,
    // replayed many times, walks every phase the budget allows
    const double tPlanned = host_ms();
    b.st.stage(c, plans, phases, true, b.stream, b.walkBudget, !keepPlans);
    b.hostPlanMs = tPlanned - tStart;
    b.hostStageMs = host_ms() - tPlanned;
}

// Each rule's support and body size after a run: static values, the plans'
// own counts (shared ones included) and fused support counts.
void phase_counts(const Batch& b, std::vector<int64_t>& sup, std::vector<int64_t>& body) {
    sup.resize(b.n);
    body.resize(b.n);
    for (int i = 0; i < b.n; ++i) { sup[i] = b.rps[i].support.value; body[i] = b.rps[i].body.value; }
    const unsigned long long* cnt = b.st.counts();
    for (size_t k = 0; k < b.owner.size(); ++k) {
        int i = b.owner[k] / 2;
        if (b.owner[k] % 2 == 0) sup[i] = (int64_t)cnt[k];
        else body[i] = (int64_t)cnt[k];
    }
    for (const auto& sh : b.shared) {
        int i = sh.first / 2;
        if (sh.first % 2 == 0) sup[i] = (int64_t)cnt[sh.second];
        else body[i] = (int64_t)cnt[sh.second];
    }
    for (int i = 0; i < b.n && i < (int)b.supOf.size(); ++i)
        if (b.supOf[i] >= 0) sup[i] = (int64_t)cnt[b.supOf[i]];
}

void collect(const Batch& b, GpuRuleResult* out, int* status) {
    std::vector<int64_t> sup, body;
    phase_counts(b, sup, body);
    for (int i = 0; i < b.n; ++i) {
        if (status) status[i] = b.parseStatus[i];
        if (b.parseStatus[i] != 0) { out[i] = GpuRuleResult{}; continue; }
        compose(b.rps[i], sup[i], body[i], 0.0, 0.0, &out[i]);
    }
}

// Runs a prepared batch: optional L2 flush (untimed), then the device work
// between two events, then the result download.
void drop_graph(Batch& b) {
    if (b.exec) { cudaGraphExecDestroy(b.exec); b.exec = nullptr; }
    if (b.graph) { cudaGraphDestroy(b.graph); b.graph = nullptr; }
}

void run_batch(Batch& b, bool useGraph, size_t flushBytes, bool retried = false) {
    Context& c = *b.c;
    if (flushBytes) {
        b.flush.ensure(flushBytes);
        ck(cudaMemsetAsync(b.flush.p, (int)(b.lastMs * 7) & 0xff, flushBytes, b.stream), "flush");
    }
    if (useGraph && !b.exec && b.st.nPlans) {
        ck(cudaStreamBeginCapture(b.stream, cudaStreamCaptureModeThreadLocal), "capture");
        b.st.enqueue(c, b.stream, 0);
        ck(cudaStreamEndCapture(b.stream, &b.graph), "capture end");
        ck(cudaGraphInstantiate(&b.exec, b.graph, 0), "graph instantiate");
    }
    ck(cudaEventRecord(b.ev0, b.stream), "event");
    if (useGraph && b.exec) ck(cudaGraphLaunch(b.exec, b.stream), "graph launch");
    else b.st.enqueue(c, b.stream, 0);
    ck(cudaEventRecord(b.ev1, b.stream), "event");
    b.st.download(b.stream);
    ck(cudaStreamSynchronize(b.stream), "engine");
    b.st.check_status();
    if (!retried && b.st.sort_overflow()) {
        // sort-mode keys outgrew the estimate: stage again with the exact
        // count (the next runs fit) and run once more
        b.st.restage(c, b.stream);
        drop_graph(b);
        run_batch(b, useGraph, flushBytes, true);
        return;
    }
    float ms = 0.f;
    ck(cudaEventElapsedTime(&ms, b.ev0, b.ev1), "elapsed");
    b.lastMs = ms;
}

Context* as_ctx(void* p) { return static_cast<Context*>(p); }

}  // namespace
}  // namespace gr

using namespace gr;

namespace {

// The rest of a load, whichever source the index came from: the state built
// on the index, and its upload.
void finish_load(Context* c) {
    // GPU_RULES_MEMO3=0 switches the three-step suffix memos off,
    // GPU_RULES_FUSE_SUPPORT=0 the fused support of batches,
    // GPU_RULES_HUB_CLAIMS=0 the skipping of repeated leaf hub items
    if (const char* m = std::getenv("GPU_RULES_MEMO3")) c->memo3 = std::atoi(m) != 0;
    if (const char* f = std::getenv("GPU_RULES_FUSE_SUPPORT")) c->fuseSupport = std::atoi(f) != 0;
    if (const char* h = std::getenv("GPU_RULES_HUB_CLAIMS")) c->hubClaims = std::atoi(h) != 0;
    // GPU_RULES_HOST_PROFILE=1: one stderr line of host-side times per one-shot batch
    if (const char* h = std::getenv("GPU_RULES_HOST_PROFILE")) c->hostProfile = std::atoi(h) != 0;
    c->tasks.reset(new TaskBuilder(c->hix));
    c->tasks->memoRows = [c](int p1, int d1, int p2, int d2, int p3, int d3,
                             double* cost) -> const std::vector<uint8_t>* {
        auto it = c->memos.find(memo_key(p1, d1, p2, d2, p3, d3));
        if (it == c->memos.end() || !it->second) return nullptr;
        // a memo word costs about a quarter of a candidate; an item itself is
        // a chain of dependent loads on one warp (exception lookups, searches
        // of the hub row for bound values; a three-step item also looks up
        // the rows its root reaches): c3 rule 963 (two steps, 4-word memos)
        // measured ~12 us of block time per root against ~7 ns per candidate
        *cost = it->second->words / 4.0 + (p3 >= 0 ? 512.0 : 256.0);
        return &it->second->rowHasMemo;
    };
    c->parser.reset(new RuleParser(c->ents, c->preds, c->prefixes));
    c->init_device();
    c->upload_index();
}

}  // namespace

extern "C" {

const char* gpu_last_error(void) { return g_lastError.c_str(); }

int gpu_query_vram(size_t* freeBytesOut, size_t* totalBytesOut) {
    size_t f = 0, t = 0;
    if (cudaMemGetInfo(&f, &t) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    if (freeBytesOut) *freeBytesOut = f;
    if (totalBytesOut) *totalBytesOut = t;
    return 0;
}

void* gpu_load_graph(const char* ttlPath) {
    if (!ttlPath) { set_error("gpu_load_graph: null path"); return nullptr; }
    Context* c = nullptr;
    try {
        c = new Context();
        std::vector<int32_t> spo;
        std::string err, text;
        if (!read_file(ttlPath, text, &err)) {
            set_error("Failed to parse TTL: " + std::string(ttlPath) + " (" + err + ")");
            delete c;
            return nullptr;
        }
        // one read of the file: the triples (several threads) and the rule
        // parser's prefix lines come from the same text
        parse_turtle_text_parallel(text, c->ents, c->preds, spo);
        c->prefixes = scan_rule_prefixes_text(text);
        std::string().swap(text);
        // GPU_RULES_MEMO_GAIN overrides the suffix-memo threshold (negative: no memos)
        if (const char* g = std::getenv("GPU_RULES_MEMO_GAIN")) c->memoGain = std::atof(g);
        // GPU_RULES_HUB_MIN_DEGREE overrides the hub-row threshold (0: no hub rows)
        int32_t hubMin = kHubMinDegree;
        if (const char* h = std::getenv("GPU_RULES_HUB_MIN_DEGREE")) hubMin = std::max(0, std::atoi(h));
        // the index is built on the device (GPU_RULES_INDEX_BUILD=host: on host threads)
        const char* where = std::getenv("GPU_RULES_INDEX_BUILD");
        if (where && std::strcmp(where, "host") == 0)
            c->hix = build_index(spo, (int32_t)c->ents.size(), (int32_t)c->preds.size(), hubMin);
        else
            c->hix = build_index_device(spo, (int32_t)c->ents.size(), (int32_t)c->preds.size(), hubMin);
        finish_load(c);
        return c;
    } catch (const std::exception& e) {
        set_error(std::string("gpu_load_graph error: ") + e.what());
        cudaGetLastError();
        delete c;
        return nullptr;
    }
}

void* gpu_load_index(const char* path) {
    if (!path) { set_error("gpu_load_index: null path"); return nullptr; }
    Context* c = nullptr;
    try {
        c = new Context();
        std::string err;
        if (!load_graph_file(path, c->ents, c->preds, c->prefixes, c->hix, &err)) {
            set_error(err);
            delete c;
            return nullptr;
        }
        if (const char* g = std::getenv("GPU_RULES_MEMO_GAIN")) c->memoGain = std::atof(g);
        finish_load(c);
        return c;
    } catch (const std::exception& e) {
        set_error(std::string("gpu_load_index error: ") + e.what());
        cudaGetLastError();
        delete c;
        return nullptr;
    }
}

int gpu_save_index(void* ctx, const char* path) {
    if (!ctx || !path) return -1;
    Context& c = *as_ctx(ctx);
    std::string err;
    if (!save_graph_file(path, c.ents, c.preds, c.prefixes, c.hix, &err)) {
        set_error(err);
        return -1;
    }
    return 0;
}

void gpu_free_graph(void* ctx) {
    if (!ctx) return;
    delete as_ctx(ctx);
}

int gpu_evaluate_rule(void* ctx, const char* ruleText, GpuRuleResult* out) {
    if (!ctx || !ruleText || !out) return -1;
    *out = GpuRuleResult{};
    Context& c = *as_ctx(ctx);
    try {
        cudaSetDevice(c.device);
        Rule r = c.parser->parse_text(ruleText);
        return evaluate_parsed(c, r, out);
    } catch (const std::exception& e) {
        set_error(std::string("gpu_evaluate_rule error: ") + e.what());
        *out = GpuRuleResult{};
        return -1;
    }
}

int gpu_evaluate_rule_json(void* ctx, const char* ruleJson, GpuRuleResult* out) {
    if (!ctx || !ruleJson || !out) return -1;
    *out = GpuRuleResult{};
    Context& c = *as_ctx(ctx);
    try {
        cudaSetDevice(c.device);
        Rule r = c.parser->parse_json(ruleJson);
        return evaluate_parsed(c, r, out);
    } catch (const std::exception& e) {
        set_error(std::string("gpu_evaluate_rule_json error: ") + e.what());
        *out = GpuRuleResult{};
        return -1;
    }
}

int gpu_evaluate_rules_batch(void* ctx, const char* const* rules, int n, int isJson,
                             GpuRuleResult* out, int* status, double* deviceMs) {
    if (!ctx || n < 0 || (n > 0 && (!rules || !out))) return -1;
    Context& c = *as_ctx(ctx);
    if (deviceMs) *deviceMs = 0.0;
    try {
        cudaSetDevice(c.device);
        // Pipelined: chunk k+1 is parsed, planned and staged on the host
        // while chunk k runs on the device (each chunk on its own stream).
        // automatic: up to 6 chunks of at least 1,667 rules (c3, 10,000 rules:
        // 1, 2, 4, 6, 8 and 12 chunks measured 53.6, 36.3, 29.0, 27.8, 30.0
        // and 34.1 ms a call)
        const int K = c.batchChunks > 0 ? std::max(1, std::min(c.batchChunks, std::max(n, 1)))
                                        : std::max(1, std::min(6, (n + 1666) / 1667));
        while ((int)c.pipe.size() < K) c.pipe.push_back(new Batch());
        const double t0 = host_ms();
        double planMs = 0, stageMs = 0;
        for (int k = 0; k < K; ++k) {
            const int lo = (int)((long long)n * k / K), hi = (int)((long long)n * (k + 1) / K);
            Batch& b = *c.pipe[k];
            prepare(b, c, rules + lo, hi - lo, isJson, false);
            planMs += b.hostPlanMs;
            stageMs += b.hostStageMs;
            ck(cudaEventRecord(b.ev0, b.stream), "event");
            b.st.enqueue(c, b.stream, 0);
            ck(cudaEventRecord(b.ev1, b.stream), "event");
            b.st.download(b.stream);
        }
        const double t1 = host_ms();
        float span = 0.f;
        for (int k = 0; k < K; ++k) {
            Batch& b = *c.pipe[k];
            ck(cudaStreamSynchronize(b.stream), "engine");
            b.st.check_status();
            if (b.st.sort_overflow()) {   // run this chunk again with the exact key count
                b.st.restage(c, b.stream);
                ck(cudaEventRecord(b.ev0, b.stream), "event");
                b.st.enqueue(c, b.stream, 0);
                ck(cudaEventRecord(b.ev1, b.stream), "event");
                b.st.download(b.stream);
                ck(cudaStreamSynchronize(b.stream), "engine");
                b.st.check_status();
            }
            float ms = 0.f;
            ck(cudaEventElapsedTime(&ms, c.pipe[0]->ev0, b.ev1), "elapsed");
            span = std::max(span, ms);
            if (c.hostProfile) {
                float own = 0.f, at = 0.f;
                ck(cudaEventElapsedTime(&own, b.ev0, b.ev1), "elapsed");
                ck(cudaEventElapsedTime(&at, c.pipe[0]->ev0, b.ev0), "elapsed");
                std::fprintf(stderr, "[gpu_rules]   chunk %d: %d rules, %d tasks, enqueued at %.2f ms, %.2f ms on the device\n",
                             k, b.n, b.st.nTasks, (double)at, (double)own);
            }
            const int lo = (int)((long long)n * k / K);
            collect(b, out + lo, status ? status + lo : nullptr);
        }
        if (deviceMs) *deviceMs = span;
        if (c.hostProfile) {
            double sect[6] = {0, 0, 0, 0, 0, 0};
            for (int k = 0; k < K; ++k)
                for (int j = 0; j < 6; ++j) {
                    sect[j] += c.pipe[k]->st.hostSect[j];
                    c.pipe[k]->st.hostSect[j] = 0.0;
                }
            std::fprintf(stderr, "[gpu_rules] batch of %d in %d chunks: parse+plan %.2f ms, staging %.2f ms "
                         "(dedup %.2f, memos %.2f, tasks %.2f, plans %.2f, order %.2f, upload %.2f), enqueue loop "
                         "%.2f ms, wait+collect %.2f ms, device span %.2f ms\n",
                         n, K, planMs, stageMs, sect[0], sect[1], sect[2], sect[3], sect[4], sect[5],
                         t1 - t0 - planMs - stageMs, host_ms() - t1, (double)span);
        }
        return 0;
    } catch (const std::exception& e) {
        set_error(std::string("gpu_evaluate_rules_batch error: ") + e.what());
        // no chunk may still be writing into the reused buffers, and the
        // caller sees no partial results
        for (Batch* b : c.pipe)
            if (b && b->stream) cudaStreamSynchronize(b->stream);
        cudaGetLastError();
        for (int i = 0; i < n; ++i) {
            out[i] = GpuRuleResult{};
            if (status) status[i] = -1;
        }
        return -1;
    }
}

void* gpu_batch_prepare(void* ctx, const char* const* rules, int n, int isJson) {
    if (!ctx || n < 0 || (n > 0 && !rules)) return nullptr;
    Context& c = *as_ctx(ctx);
    Batch* b = nullptr;
    try {
        cudaSetDevice(c.device);
        b = new Batch();
        b->walkBudget = 4.0e7;   // prepared once, replayed many times
        prepare(*b, c, rules, n, isJson);
        ck(cudaStreamSynchronize(b->stream), "stage");
        return b;
    } catch (const std::exception& e) {
        set_error(std::string("gpu_batch_prepare error: ") + e.what());
        delete b;
        return nullptr;
    }
}

int gpu_batch_run(void* batch, long long flushBytes, GpuRuleResult* out, int* status, double* deviceMs) {
    if (!batch) return -1;
    Batch& b = *static_cast<Batch*>(batch);
    try {
        cudaSetDevice(b.c->device);
        run_batch(b, true, flushBytes > 0 ? (size_t)flushBytes : 0);
        if (out) collect(b, out, status);
        if (deviceMs) *deviceMs = b.lastMs;
        return 0;
    } catch (const std::exception& e) {
        set_error(std::string("gpu_batch_run error: ") + e.what());
        return -1;
    }
}

int gpu_batch_counts(void* batch, long long* counts, int* status) {
    if (!batch || !counts) return -1;
    const Batch& b = *static_cast<const Batch*>(batch);
    std::vector<int64_t> sup, body;
    phase_counts(b, sup, body);
    for (int i = 0; i < b.n; ++i) {
        const RulePlan& rp = b.rps[i];
        const bool ok = b.parseStatus[i] == 0;
        const bool run = ok && rp.status == kRuleOk;
        counts[4 * i + 0] = run ? sup[i] : 0;
        counts[4 * i + 1] = ok ? rp.headSize : 0;
        counts[4 * i + 2] = ok ? rp.headSupport : 0;
        counts[4 * i + 3] = run ? body[i] : 0;
        if (status) status[i] = b.parseStatus[i];
    }
    return 0;
}

int gpu_evaluate_rule_shard(void* ctx, const char* ruleText, int shard, int nShards, long long* counts) {
    if (!ctx || !ruleText || !counts || nShards < 1 || shard < 0 || shard >= nShards) return -1;
    Context& c = *static_cast<Context*>(ctx);
    try {
        cudaSetDevice(c.device);
        evaluate_shard(c, c.parser->parse_text(ruleText), shard, nShards, counts);
        return 0;
    } catch (const std::exception& e) {
        set_error(std::string("gpu_evaluate_rule_shard error: ") + e.what());
        return -1;
    }
}

int gpu_batch_info(void* batch, long long* plans, long long* tasks, long long* h2dBytes, long long* d2hBytes) {
    if (!batch) return -1;
    Batch& b = *static_cast<Batch*>(batch);
    if (plans) *plans = b.st.nPlans;
    if (tasks) *tasks = b.st.nTasks;
    if (h2dBytes) *h2dBytes = (long long)b.st.h2dBytes;
    if (d2hBytes) *d2hBytes = (long long)b.st.d2hBytes;
    return 0;
}

int gpu_batch_kernels(void* batch) {
    if (!batch) return -1;
    return static_cast<const Batch*>(batch)->st.kernels_per_enqueue();
}

int gpu_batch_dedup(void* batch, int* modes, long long* sortKeys) {
    if (!batch || !modes) return -1;
    const Batch& b = *static_cast<const Batch*>(batch);
    for (int i = 0; i < b.n; ++i) modes[i] = -1;
    // the body-size phase (owner rule * 2 + 1) of each rule whose body size
    // counts pairs on the device
    auto put = [&](int owner, int plan) {
        if (owner % 2 != 1 || plan < 0 || plan >= (int)b.st.dedup.size() || plan >= (int)b.phases.size()) return;
        if (b.phases[plan]->plan.mode == kPairs) modes[owner / 2] = b.st.dedup[plan];
    };
    for (size_t k = 0; k < b.owner.size(); ++k) put(b.owner[k], (int)k);
    for (const auto& sh : b.shared) put(sh.first, sh.second);
    if (sortKeys) *sortKeys = b.st.nSort ? (long long)*static_cast<const unsigned long long*>(b.st.hSort.p) : 0;
    return 0;
}

int gpu_batch_count_bytes(void* batch, unsigned long long* bytes) {
    return gpu_batch_profile(batch, bytes, nullptr, nullptr, 0);
}

int gpu_batch_profile(void* batch, unsigned long long* bytes, unsigned long long* taskNs, int* taskInfo,
                      long long maxTasks) {
    if (!batch) return -1;
    Batch& b = *static_cast<Batch*>(batch);
    try {
        cudaSetDevice(b.c->device);
        if (bytes) *bytes = 0;
        if (!b.st.nPlans) return 0;
        b.st.enqueue(*b.c, b.stream, 2);
        unsigned long long by = 0;
        ck(cudaMemcpyAsync(&by, b.st.dBytes.p, 8, cudaMemcpyDeviceToHost, b.stream), "D2H bytes");
        long long n = std::min<long long>(maxTasks, b.st.nTasks);
        if (taskNs && n > 0)
            ck(cudaMemcpyAsync(taskNs, b.st.dTaskNs.p, (size_t)n * 16, cudaMemcpyDeviceToHost, b.stream), "D2H task times");
        ck(cudaStreamSynchronize(b.stream), "profile");
        if (bytes) *bytes = by;
        if (taskInfo)
            for (long long t = 0; t < n; ++t) {
                const DevTask& tk = b.st.hTasks[t];
                taskInfo[3 * t] = b.owner[tk.plan];
                taskInfo[3 * t + 1] = tk.beg;
                taskInfo[3 * t + 2] = tk.end;
            }
        return 0;
    } catch (const std::exception& e) {
        set_error(std::string("gpu_batch_profile error: ") + e.what());
        return -1;
    }
}

int gpu_batch_autotune(void* batch, int rounds) {
    if (!batch || rounds < 0) return -1;
    Batch& b = *static_cast<Batch*>(batch);
    try {
        Context& c = *b.c;
        cudaSetDevice(c.device);
        for (int r = 0; r < rounds && b.st.nPlans; ++r) {
            b.st.enqueue(c, b.stream, 1);
            std::vector<unsigned long long> ns(2 * (size_t)b.st.nTasks);
            ck(cudaMemcpyAsync(ns.data(), b.st.dTaskNs.p, ns.size() * 8, cudaMemcpyDeviceToHost, b.stream), "D2H task times");
            ck(cudaStreamSynchronize(b.stream), "autotune");
            c.tasks->learn(b.phases, b.st.hTasks, b.st.hCost, ns.data(), c.grid);
            drop_graph(b);
            std::vector<DevPlan> pl = b.plans0;
            b.st.stage(c, pl, b.phases, true, b.stream, b.walkBudget);
            ck(cudaStreamSynchronize(b.stream), "restage");
        }
        return 0;
    } catch (const std::exception& e) {
        set_error(std::string("gpu_batch_autotune error: ") + e.what());
        return -1;
    }
}

int gpu_set_option(void* ctx, const char* name, long long value) {
    if (!ctx || !name) return -1;
    Context& c = *as_ctx(ctx);
    std::string n(name);
    if (n == "block") return c.set_block((int)value) ? 0 : -1;
    if (n == "task_target" && value >= 0) { c.tasks->forceTarget = (double)value; return 0; }
    if (n == "walk_threshold" && value >= 0) { c.tasks->walkThreshold = (double)value; return 0; }
    if (n == "serve_lanes" && (value == 0 || value == 1)) { c.serveLanes = (int)value; return 0; }
    if (n == "rule_walk_budget" && value >= 0) { c.ruleWalkBudget = (double)value; return 0; }
    if (n == "batch_chunks" && value >= 0 && value <= 16) { c.batchChunks = (int)value; return 0; }
    if (n == "rule_block" && (value == 0 || value == 128 || value == 256 || value == 512)) {
        c.ruleBlock = (int)value;
        return 0;
    }
    if (n == "serve_heavy_share" && value >= 1 && value <= 16) { c.serveHeavyShare = (int)value; return 0; }
    if (n == "serve_heavy_us" && value >= 0) { c.serveHeavyNs = 1e3 * (double)value; return 0; }
    if (n == "serve_deadline_us" && value >= 0) { c.serveDeadlineNs = 1e3 * (double)value; return 0; }
    if (n == "serve_max_us" && value >= 0) { c.serveMaxNs = 1e3 * (double)value; return 0; }
    if (n == "batch_phases" && value >= 1 && value <= 3) { c.batchPhases = (int)value; return 0; }
    if (n == "dedup_budget" && value >= 4096) { c.dedupBudget = (size_t)value; return 0; }
    if (n == "dedup_mode" && (value == 0 || value == kDedupRows || value == kDedupBlockRows || value == kDedupSort)) {
        c.dedupForce = (int)value;
        return 0;
    }
    return -1;
}

void gpu_batch_free(void* batch) {
    delete static_cast<Batch*>(batch);
}

int gpu_graph_stats(void* ctx, long long* entities, long long* predicates, long long* triples) {
    if (!ctx) return -1;
    Context& c = *as_ctx(ctx);
    if (entities) *entities = (long long)c.hix.nEnt;
    if (predicates) *predicates = (long long)c.hix.nPred;
    if (triples) *triples = (long long)c.hix.nTriples;
    return 0;
}

int gpu_graph_predicate(void* ctx, long long index, char* name, int capacity, long long* triples) {
    if (!ctx) return -1;
    Context& c = *as_ctx(ctx);
    if (index < 0 || index >= (long long)c.preds.size()) return -1;
    const std::string& s = c.preds.names[(size_t)index];
    if (triples) *triples = (long long)c.hix.pred_size((int32_t)index);
    if (name && capacity > 0) {
        const size_t n = std::min(s.size(), (size_t)capacity - 1);
        std::memcpy(name, s.data(), n);
        name[n] = 0;
    }
    return (int)s.size();
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Evaluation without device allocation.
//
// Some callers cannot call cudaMalloc while they evaluate rules: a host
// framework that owns a fixed device-memory budget and forbids allocation at
// request time, a serving loop that must not hit cudaMalloc/cudaFree (both can
// synchronise the whole device and stall concurrent work), or code that runs
// between other libraries' stream-ordered work and must not change the
// device's memory map.  gpu_evaluate_rule_noalloc serves them: it evaluates a
// rule exactly like gpu_evaluate_rule (one launch per phase, same results)
// but takes every per-call device buffer (plan, tasks, task counter, status
// word, result counter and, for very large hO domains, the pair bitmap) from
// the fixed array below instead of allocating.
//
// The array is a file-scope __device__ object of kNoAllocScratchBytes; every
// GPU that loads this library holds it until the process exits.  Host code
// cannot use the array's name as a device address, so the first call on each
// device (with that device current) looks the address up with
// cudaGetSymbolAddress and caches it; make that first call before any stream
// capture.  All calls share the array and it keeps the previous call's
// contents, so each call clears the parts that must start at zero.  Calls
// that overlap on the GPU (from several threads, contexts or streams of the
// same device) race on the array and must be serialised by the caller.
namespace gr {
namespace {
constexpr size_t kNoAllocScratchBytes = 8u << 20;   // 8 MiB
constexpr size_t kNoAllocHeader = 256;               // [0,8) counter+status, [64,72) result
constexpr int kNoAllocMaxDevices = 64;
}  // namespace
}  // namespace gr

static __device__ __align__(256) unsigned char g_noallocScratch[gr::kNoAllocScratchBytes];

namespace gr {
namespace {

std::mutex g_noallocMu;
void* g_noallocAddr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on `dev` (which must be current).
void* noalloc_scratch(int dev) {
    if (dev < 0 || dev >= kNoAllocMaxDevices) throw CudaError("device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_noallocMu);
    if (!g_noallocAddr[dev]) {
        void* p = nullptr;
        ck(cudaGetSymbolAddress(&p, g_noallocScratch), "cudaGetSymbolAddress(scratch)");
        g_noallocAddr[dev] = p;
    }
    return g_noallocAddr[dev];
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

int64_t run_phase_noalloc(Context& c, const PhasePlan& ph, char* scratch, float* ms) {
    DevPlan plan = ph.plan;
    std::vector<PhaseTasks> pts;
    c.tasks->build({&ph}, c.grid, false, pts);
    std::vector<DevTask>& tasks = pts[0].tasks;
    const size_t planOff = kNoAllocHeader;
    const size_t taskOff = align256(planOff + sizeof(DevPlan));
    const size_t bitmapOff = align256(taskOff + tasks.size() * sizeof(DevTask));
    size_t bitmapWords = 0;
    if (ph.needsGlobalBitmap)
        bitmapWords = (size_t)(ph.rootEnd - ph.rootBeg) * (size_t)std::max(plan.rowWords, 1);
    const size_t need = bitmapOff + bitmapWords * 4;
    if (need > kNoAllocScratchBytes)
        throw CudaError("rule needs " + std::to_string(need) + " bytes of scratch; the no-allocation limit is " +
                        std::to_string(kNoAllocScratchBytes) + " bytes");
    plan.resultSlot = 0;
    plan.gBitmap = bitmapWords ? reinterpret_cast<uint32_t*>(scratch + bitmapOff) : nullptr;
    plan.gRowBase = bitmapWords ? ph.rootBeg : 0;
    int* ctl = reinterpret_cast<int*>(scratch);
    unsigned long long* result = reinterpret_cast<unsigned long long*>(scratch + 64);
    ck(cudaMemcpyAsync(scratch + planOff, &plan, sizeof(DevPlan), cudaMemcpyHostToDevice, c.stream), "H2D plan");
    if (!tasks.empty())
        ck(cudaMemcpyAsync(scratch + taskOff, tasks.data(), tasks.size() * sizeof(DevTask), cudaMemcpyHostToDevice,
                           c.stream), "H2D tasks");
    ck(cudaMemsetAsync(scratch, 0, kNoAllocHeader, c.stream), "clear header");
    if (bitmapWords) ck(cudaMemsetAsync(scratch + bitmapOff, 0, bitmapWords * 4, c.stream), "clear bitmap");
    ck(cudaEventRecord(c.ev[2], c.stream), "event");
    int grid = std::max(1, std::min((int)tasks.size(), c.grid));
    ck(engine_launch(c.dix, reinterpret_cast<const DevPlan*>(scratch + planOff),
                     reinterpret_cast<const DevTask*>(scratch + taskOff), (int)tasks.size(), ctl, result, ctl + 1,
                     grid, c.geom.block, c.stream, nullptr), "engine launch");
    ck(cudaEventRecord(c.ev[3], c.stream), "event");
    unsigned long long count = 0;
    int st[2] = {0, 0};
    ck(cudaMemcpyAsync(&count, result, sizeof(count), cudaMemcpyDeviceToHost, c.stream), "D2H result");
    ck(cudaMemcpyAsync(st, ctl, sizeof(st), cudaMemcpyDeviceToHost, c.stream), "D2H status");
    ck(cudaStreamSynchronize(c.stream), "engine");
    if (st[1] != 0) throw CudaError("engine reported internal status " + std::to_string(st[1]));
    ck(cudaEventElapsedTime(ms, c.ev[2], c.ev[3]), "elapsed");
    return (int64_t)count;
}

}  // namespace
}  // namespace gr

extern "C" int gpu_evaluate_rule_noalloc(void* ctx, const char* ruleText, GpuRuleResult* out) {
    if (!ctx || !ruleText || !out) return -1;
    *out = GpuRuleResult{};
    Context& c = *as_ctx(ctx);
    try {
        ck(cudaSetDevice(c.device), "cudaSetDevice");
        char* scratch = static_cast<char*>(noalloc_scratch(c.device));
        Rule r = c.parser->parse_text(ruleText);
        RulePlan rp = plan_rule(r, c.hix, c.geom);
        int64_t sup = rp.support.value, body = rp.body.value;
        float supMs = 0.f, confMs = 0.f;
        if (rp.status == kRuleOk && rp.support.how == kDevice) sup = run_phase_noalloc(c, rp.support, scratch, &supMs);
        if (rp.status == kRuleOk && rp.body.how == kDevice) body = run_phase_noalloc(c, rp.body, scratch, &confMs);
        compose(rp, sup, body, supMs, confMs, out);
        return 0;
    } catch (const std::exception& e) {
        set_error(std::string("gpu_evaluate_rule_noalloc error: ") + e.what());
        *out = GpuRuleResult{};
        return -1;
    }
}
