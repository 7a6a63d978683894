// engine.hpp — host-side engine state shared by the C ABI (context.cu) and
// the serving loop (serve.cu): device buffers, staged launches, the graph
// context and prepared batches.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <climits>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/gpu_rules_api.h"
#include "common.hpp"
#include "index.hpp"
#include "planner.hpp"
#include "rules.hpp"
#include "tasks.hpp"
#include "turtle.hpp"

namespace gr {

size_t engine_smem_bytes(int block);
cudaError_t engine_configure();
// maxWo: the largest three-step domain among the jobs (0: none), which
// sizes the shared path counters.
cudaError_t memo_build(const DevIndex& ix, const MemoJob* jobs, int nJobs, int maxWo, cudaStream_t stream);
// Fused support of split heavy roots, after the engine launch that filled
// their rows (see DevPlan::supN).
cudaError_t support_rows(const DevIndex& ix, const DevPlan* plans, const SupJob* jobs, int nJobs,
                         unsigned long long* results, cudaStream_t stream);
cudaError_t engine_launch(const DevIndex& ix, const DevPlan* plans, const DevTask* tasks, int nTasks,
                          int* taskCounter, unsigned long long* results, int* status, int grid, int block,
                          cudaStream_t stream, const EngineProfile* prof);
// Sort mode (sort.cu): radix sort of the appended pair keys and the count of
// each plan's distinct keys into its result slot.
size_t pairs_sort_hist_words(unsigned long long cap);
// Sorts min(*count, cap) keys by their low `bits` bits (8 bits a pass,
// stable), ping-ponging with tmp; returns the buffer that holds the result.
unsigned long long* radix_sort_keys(unsigned long long* keys, unsigned long long* tmp, const unsigned long long* count,
                                    unsigned long long cap, int bits, uint32_t* hist, int grid, cudaStream_t stream,
                                    cudaError_t* err);
cudaError_t pairs_sort_count(unsigned long long* keys, unsigned long long* tmp, const unsigned long long* count,
                             unsigned long long cap, int bits, int slotShift, const int32_t* slotOf, int nSlots,
                             unsigned long long* results, int* status, uint32_t* hist, int grid,
                             cudaStream_t stream);

// Records the calling thread's last error (gpu_last_error) and logs it.
void set_error(const std::string& s);

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

inline void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    bool pooled = false;   // from the stream-ordered allocator
    // Grows by half again: cudaFree synchronises the device, so resizing
    // must be rare when request sizes vary.  With a stream, the old buffer
    // is freed and the new one allocated in that stream's order (no device
    // synchronisation); the buffer must then only be used on that stream.
    void ensure(size_t bytes, cudaStream_t s = nullptr) {
        if (bytes <= cap) return;
        size_t want = std::max<size_t>(bytes + bytes / 2, 4096);
        if (s) {
            if (p && pooled) ck(cudaFreeAsync(p, s), "cudaFreeAsync");
            else release();
            p = nullptr;
            cap = 0;
            ck(cudaMallocAsync(&p, want, s), "cudaMallocAsync");
            pooled = true;
        } else {
            release();
            ck(cudaMalloc(&p, want), "cudaMalloc");
            pooled = false;
        }
        cap = want;
    }
    void release() {
        if (p) cudaFree(p);   // also frees pooled memory, after a synchronisation
        p = nullptr;
        cap = 0;
    }
    ~DevBuf() { release(); }
};

struct HostBuf {  // pinned
    void* p = nullptr;
    size_t cap = 0;
    void ensure(size_t bytes) {
        if (bytes <= cap) return;
        release();
        size_t want = std::max<size_t>(bytes + bytes / 2, 4096);
        ck(cudaMallocHost(&p, want), "cudaMallocHost");
        cap = want;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
    }
    ~HostBuf() { release(); }
};

inline int64_t clamp_int(int64_t v) { return std::min<int64_t>(v, INT_MAX); }

struct Context;

// A set of plans and their tasks resident on the device, with the buffers
// one launch over them needs.
struct Staged {
    DevBuf dBlob, dResults, dCtl, dBitmap, dHeavy, dBytes, dTaskNs, dSort, dIncomplete;
    std::vector<DevTask> hTasks;  // task list as uploaded (for profiles)
    std::vector<double> hCost;    // estimated work per uploaded task
    HostBuf hBlob, hResults, hCtl;
    const DevPlan* dPlans = nullptr;
    const DevTask* dTasks = nullptr;
    int nPlans = 0, nTasks = 0;
    size_t bitmapWords = 0, heavyWords = 0;
    size_t h2dBytes = 0, d2hBytes = 0;
    bool streamOrdered = false;   // grow device buffers on the launch stream (serving slots)
    std::vector<int32_t> planTaskEnd;   // tasks in plan order (unsorted staging): end of each plan's tasks

    // Deduplication of kPairs plans (DedupMode per plan).  Per-phase global
    // rows while all of them fit the context's budget; beyond it, per plan,
    // block rows (each resident block owns `blockWords` words after the
    // per-phase rows in dBitmap, `blockRegions` regions) or sort mode (keys
    // in dSort: [cursor | keys | tmp | histogram]), whichever the byte
    // estimate favours.
    std::vector<int32_t> dedup;
    size_t blockWords = 0, blockRegions = 0;
    int nSort = 0, sortBits = 0, sortSlotShift = 0;
    unsigned long long keyCap = 0;
    unsigned long long keyHint = 0;     // exact keys of a run that overflowed keyCap
    const int32_t* dSortSlots = nullptr;   // result slot of each sort index (in dBlob)
    // Result slots after the plans' own (fused support counts, see
    // RulePlan::supFuse), set before staging; nResults = nPlans + extraResults.
    int extraResults = 0;
    int nResults = 0;
    int nSupJobs = 0;
    const SupJob* dSupJobs = nullptr;      // in dBlob
    DevBuf dHubSeen;                       // leaf hub claims: kHubSeen words per resident block
    // host ms of the staging sections (dedup and fusion, memos, task build,
    // plan fields, task order, upload), summed until read
    double hostSect[6] = {0, 0, 0, 0, 0, 0};
    HostBuf hSort;                      // the downloaded append cursor
    HostBuf hIncomplete;                // per plan: a task was abandoned at the deadline
    bool budgeted = false;              // the last enqueue ran under a deadline
    // inputs of the last staging, kept while it has sort-mode plans so that
    // an overflowing run can be staged again with the exact key count
    std::vector<DevPlan> inPlans;
    std::vector<const PhasePlan*> inPhases;
    bool inSortTasks = true, inCostAware = false, inAllowSort = true;
    double inWalk = 4.0e6;

    // walkBudget: how much per-root measurement the task builder may do
    // (prepared batches afford more than one-shot or served launches).
    // allowSort: sort mode may be chosen (launches that can be run again
    // when the key buffer overflows; the serving loop cannot).
    void stage(Context& c, std::vector<DevPlan>& plans, const std::vector<const PhasePlan*>& phases,
               bool sortTasks, cudaStream_t s, double walkBudget = 4.0e6, bool costAware = false,
               bool allowSort = true);
    // After download + synchronisation: whether sort-mode keys exceeded the
    // buffer (the counts are then incomplete).  restage() stages the same
    // plans again with a buffer of the exact size (one upload, no launch).
    bool sort_overflow() const {
        return nSort > 0 && *static_cast<const unsigned long long*>(hSort.p) > keyCap;
    }
    void restage(Context& c, cudaStream_t s);
    // Kernels one enqueue() launches: the engine, the fused support of split
    // roots when there are any, and the pair sort (three kernels per 8-bit
    // pass and the count) when sort mode is staged.
    int kernels_per_enqueue() const {
        if (!nPlans) return 0;
        return (nTasks > 0 ? 1 : 0) + (nSupJobs > 0 ? 1 : 0) + (nSort ? 3 * ((sortBits + 7) / 8) + 1 : 0);
    }
    // instr: 0 plain, 1 task times into dTaskNs, 2 also algorithmic bytes
    // into dBytes.  gridCap > 0 limits the launch to that many blocks (a
    // share of the SMs).  budgetNs > 0 (with instr 1): blocks stop that long
    // after they start, and plan_incomplete() tells which plans lost work.
    void enqueue(Context& c, cudaStream_t s, int instr, int gridCap = 0, unsigned long long budgetNs = 0);
    int stagedBlock = 0;   // block size whose shared pool the staged plans are laid out for
    // Throws when the context's block size is below stagedBlock.
    void check_geometry(const Context& c) const;
    bool plan_incomplete(int i) const {
        return budgeted && static_cast<const int*>(hIncomplete.p)[i] != 0;
    }
    // One launch per plan of an unsorted staging (at most kMaxPerPlan plans),
    // each with its own task counter, launch span and result in the 64
    // control bytes (counters and status at 0, spans at 16, results at
    // kPerPlanResults), cleared by one memset; download_spans brings them
    // back in one copy.  The plain per-rule form: support and body size of
    // one rule.
    static constexpr int kMaxPerPlan = 2;
    static constexpr int kPerPlanResults = 16 + 16 * kMaxPerPlan;
    static_assert(kPerPlanResults + 8 * kMaxPerPlan <= 64, "per-plan control words fit the 64 control bytes");
    void enqueue_per_plan(Context& c, cudaStream_t s);
    void download_spans(cudaStream_t s);
    // Count of plan i after download_spans and a sync.
    unsigned long long per_plan_count(int i) const {
        return reinterpret_cast<const unsigned long long*>(static_cast<const char*>(hCtl.p) + kPerPlanResults)[i];
    }
    // Device span (ms) of plan i's launch after download_spans and a sync.
    double span_ms(int i) const {
        const unsigned long long* w = static_cast<const unsigned long long*>(hCtl.p) + 2 + 2 * i;
        const unsigned long long t0 = ~w[0], t1 = w[1];
        return t1 > t0 ? (double)(t1 - t0) * 1e-6 : 0.0;
    }
    // Pre-sizes the buffers so that launches up to this size never resize
    // (freeing device or pinned memory synchronises the whole device).
    void reserve(size_t plans, size_t tasks, cudaStream_t s = nullptr) {
        const size_t blob = plans * sizeof(DevPlan) + tasks * sizeof(DevTask);
        dBlob.ensure(blob, s);
        hBlob.ensure(blob);
        dResults.ensure(plans * sizeof(unsigned long long), s);
        hResults.ensure(plans * sizeof(unsigned long long));
        dCtl.ensure(64, s);
        hCtl.ensure(64);
        dHeavy.ensure(1 << 20, s);
        dBitmap.ensure(1 << 20, s);
        dBytes.ensure(8, s);
        dTaskNs.ensure(tasks * 16, s);
    }
    void download(cudaStream_t s) {
        if (!nPlans) return;
        ck(cudaMemcpyAsync(hResults.p, dResults.p, nResults * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s),
           "D2H results");
        ck(cudaMemcpyAsync(hCtl.p, dCtl.p, 8, cudaMemcpyDeviceToHost, s), "D2H status");
        download_cursor(s);
        if (budgeted)
            ck(cudaMemcpyAsync(hIncomplete.p, dIncomplete.p, (size_t)nPlans * sizeof(int), cudaMemcpyDeviceToHost, s),
               "D2H incomplete plans");
    }
    void download_cursor(cudaStream_t s) {
        if (nSort) ck(cudaMemcpyAsync(hSort.p, dSort.p, 8, cudaMemcpyDeviceToHost, s), "D2H key cursor");
    }
    // Sort and count the keys of the launch(es) just enqueued on s into
    // `results` (per result slot); bad keys are flagged in `status`.
    void enqueue_sort(Context& c, cudaStream_t s, unsigned long long* results, int* status);
    const unsigned long long* counts() const { return static_cast<const unsigned long long*>(hResults.p); }
    void check_status() const {
        if (nPlans && static_cast<const int*>(hCtl.p)[1] != 0)
            throw CudaError("engine reported internal status " + std::to_string(static_cast<const int*>(hCtl.p)[1]));
    }
};

// Suffix memo of one predicate transition (p1, d1) -> (p2, d2): per hub row
// of (p1, d1) worth it, the S1/S2 bitmaps over (p2, 1 - d2)'s rows (see
// memo_item in kernels.cu).  Built once per context, never moved.
constexpr size_t kMemoBudgetBytes = size_t(1) << 30;   // all suffix memos of a context

struct SuffixMemo {   // its table and bits live in one of Context::memoChunks
    const int32_t* tab = nullptr;
    const uint32_t* bits = nullptr;
    int words = 0;
    int wo = 0;          // three-step memos: ranks of the domain (one path count each)
    int slots = 0;
    std::vector<uint8_t> rowHasMemo;   // per row of (p1, d1), from the predicate's first row
};

struct Context {
    int device = 0;
    TermDict ents, preds;
    std::unordered_map<std::string, std::string> prefixes;
    HostIndex hix;
    DevBuf indexMem;
    DevIndex dix{};
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {};
    Staged one;          // per-rule launches
    std::vector<struct Batch*> pipe;  // reusable chunks of one-shot batches
    std::unique_ptr<TaskBuilder> tasks;
    Geom geom;
    double ruleWalkBudget = 4.0e6;   // per-root measurement allowed per plain per-rule launch
    int batchChunks = 0;             // pipelined chunks of one-shot batches (0: automatic)
    int batchPhases = 3;             // phases batches run on the device: 1 support, 2 body size, 3 both
    // suffix memos: a hub row gets one when its suffix candidates are at
    // least memoGain x the memo's words (negative: no memos)
    double memoGain = 0.25;
    bool memo3 = true;         // three-step suffix memos (memo3_item) for the plans that admit one
    bool fuseSupport = true;   // batches count a rule's support in its body-size plan where it can
    bool hubClaims = true;     // repeated leaf hub items of a root are skipped (see kHubSeen)
    bool hostProfile = false;  // one-shot batches print their host-side times
    std::unordered_map<uint64_t, std::unique_ptr<SuffixMemo>> memos;
    std::vector<std::unique_ptr<DevBuf>> memoChunks;   // one allocation per ensure_memos call
    size_t memoBytes = 0;
    // Builds the memos in `keys` that do not exist yet, {p1, d1, p2, d2, p3,
    // d3}: the transitions (p1, d1) -> (p2, d2), or with p3 >= 0 the
    // three-step suffixes (p1, d1) -> (p2, d2) -> (p3, d3): one kernel over
    // all their hub rows, one synchronisation of stream s (memos are shared
    // by every stream afterwards).
    void ensure_memos(const std::vector<std::array<int, 6>>& keys, cudaStream_t s);
    // The memo of a key if built, null when none exists or no hub row of
    // (p1, d1) is worth one.
    const SuffixMemo* memo_for(int p1, int d1, int p2, int d2, int p3 = -1, int d3 = 0) const;
    DevBuf memoJobs;
    int serveLanes = 1;        // servers started on this context keep a heavy lane
    int serveHeavyShare = 2;   // the heavy lane launches on grid / serveHeavyShare blocks
    double serveHeavyNs = 5.0e6;
    // servers started afterwards: a device-time budget per served launch
    // (0: none) and a limit on a request's expected device time (0: none);
    // requests beyond either complete with status -4
    double serveDeadlineNs = 0.0;
    double serveMaxNs = 0.0;
    // kPairs deduplication beyond the shared pool: device bytes that the
    // global dedup buffers of one launch may take before block rows or sort
    // mode replace per-phase rows, and a forced mode for every kPairs plan
    // (0: automatic; else a DedupMode other than kDedupShared).
    size_t dedupBudget = size_t(8) << 30;
    int dedupForce = 0;
    int grid = 0;
    int sms = 0;
    std::unique_ptr<RuleParser> parser;

    void free_pipe();
    ~Context() {
        free_pipe();
        cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        for (auto& e : ev) if (e) cudaEventDestroy(e);
        if (stream) cudaStreamDestroy(stream);
    }

    void upload_index() {
        const HostIndex& h = hix;
        std::vector<std::pair<const void*, size_t>> parts;
        auto add = [&](const void* p, size_t n) { parts.push_back({p, n}); };
        for (int d = 0; d < 2; ++d) {
            add(h.val[d].data(), h.val[d].size() * 4);
            add(h.valRank[d].data(), h.valRank[d].size() * 4);
            add(h.src[d].data(), h.src[d].size() * 4);
            add(h.srcRank[d].data(), h.srcRank[d].size() * 4);
            add(h.rowKey[d].data(), h.rowKey[d].size() * 4);
            add(h.rowBeg[d].data(), h.rowBeg[d].size() * 4);
            add(h.predRow[d].data(), h.predRow[d].size() * 4);
            add(h.predEdge[d].data(), h.predEdge[d].size() * 4);
        }
        add(h.hash.data(), h.hash.size() * sizeof(HashSlot));
        add(h.hubOf[0].data(), h.hubOf[0].size() * 4);
        add(h.hubOf[1].data(), h.hubOf[1].size() * 4);
        add(h.hubOff.data(), h.hubOff.size() * 8);
        add(h.hubBits.data(), h.hubBits.size() * 4);
        add(h.valSig[0].data(), h.valSig[0].size() * 8);
        add(h.valSig[1].data(), h.valSig[1].size() * 8);
        add(h.sufSig[0].data(), h.sufSig[0].size() * 8);
        add(h.sufSig[1].data(), h.sufSig[1].size() * 8);
        size_t total = 0;
        std::vector<size_t> off;
        for (auto& pp : parts) {
            off.push_back(total);
            total += (pp.second + 255) & ~size_t(255);
        }
        size_t freeB = 0, totB = 0;
        ck(cudaMemGetInfo(&freeB, &totB), "cudaMemGetInfo");
        if (total + (64u << 20) > freeB)
            throw CudaError("not enough device memory: need ~" + std::to_string((total >> 20) + 64) +
                            " MB, " + std::to_string(freeB >> 20) + " MB free");
        indexMem.ensure(std::max<size_t>(total, 256));
        char* base = static_cast<char*>(indexMem.p);
        for (size_t i = 0; i < parts.size(); ++i)
            if (parts[i].second)
                ck(cudaMemcpy(base + off[i], parts[i].first, parts[i].second, cudaMemcpyHostToDevice), "cudaMemcpy(index)");
        size_t k = 0;
        for (int d = 0; d < 2; ++d) {
            dix.val[d] = reinterpret_cast<const int32_t*>(base + off[k++]);
            dix.valRank[d] = reinterpret_cast<const int32_t*>(base + off[k++]);
            dix.src[d] = reinterpret_cast<const int32_t*>(base + off[k++]);
            dix.srcRank[d] = reinterpret_cast<const int32_t*>(base + off[k++]);
            dix.rowKey[d] = reinterpret_cast<const int32_t*>(base + off[k++]);
            dix.rowBeg[d] = reinterpret_cast<const int32_t*>(base + off[k++]);
            dix.predRow[d] = reinterpret_cast<const int32_t*>(base + off[k++]);
            dix.predEdge[d] = reinterpret_cast<const int32_t*>(base + off[k++]);
        }
        dix.hash = reinterpret_cast<const HashSlot*>(base + off[k++]);
        dix.hubOf[0] = reinterpret_cast<const int32_t*>(base + off[k++]);
        dix.hubOf[1] = reinterpret_cast<const int32_t*>(base + off[k++]);
        dix.hubOff = reinterpret_cast<const int64_t*>(base + off[k++]);
        dix.hubBits = reinterpret_cast<const uint32_t*>(base + off[k++]);
        dix.valSig[0] = reinterpret_cast<const uint64_t*>(base + off[k++]);
        dix.valSig[1] = reinterpret_cast<const uint64_t*>(base + off[k++]);
        dix.sufSig[0] = reinterpret_cast<const uint64_t*>(base + off[k++]);
        dix.sufSig[1] = reinterpret_cast<const uint64_t*>(base + off[k++]);
        dix.nHub = (int32_t)h.hubOff.size();
        dix.hashMask = h.hashMask;
        dix.nPred = h.nPred;
        dix.nEnt = h.nEnt;
        dix.nTriples = h.nTriples;
    }

    bool set_block(int b) {
        if (b != 128 && b != 256 && b != 512) return false;
        geom.block = b;
        grid = sms * (1024 / b);
        return true;
    }
    // Plain per-rule calls launch on 512-thread blocks: one rule has few
    // tasks, which finish sooner on larger blocks.  Their plans keep the
    // layout of geom.block.  0 (or a size not above geom.block): geom.block.
    int ruleBlock = 512;

    void init_device() {
        ck(cudaGetDevice(&device), "cudaGetDevice");
        ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "cudaDeviceGetAttribute");
        ck(engine_configure(), "cudaFuncSetAttribute");
        if (const char* b = std::getenv("GPU_RULES_BLOCK")) set_block(std::atoi(b));
        else set_block(geom.block);
        ck(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
        for (auto& e : ev) ck(cudaEventCreate(&e), "cudaEventCreate");
    }
};


// A batch prepared once and replayed: parse, plan and upload happen at
// preparation; a run is one CUDA-graph launch of the device work.
struct Batch {
    Context* c = nullptr;
    int n = 0;
    std::vector<RulePlan> rps;
    std::vector<int> parseStatus;
    std::vector<int> owner;  // plan -> rule * 2 + phase
    std::vector<int> supOf;  // rule -> result slot of its fused support count, or -1
    // phases identical to an earlier one of the batch (same plan and roots):
    // (rule * 2 + phase, plan whose count they share); computed once per run
    std::vector<std::pair<int, int>> shared;
    std::vector<DevPlan> plans0;
    std::vector<const PhasePlan*> phases;
    Staged st;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    DevBuf flush;
    double lastMs = 0.0;
    double walkBudget = 4.0e6;
    double hostPlanMs = 0.0, hostStageMs = 0.0;   // host time of the last prepare

    ~Batch() {
        if (c) cudaSetDevice(c->device);
        if (stream) cudaStreamSynchronize(stream);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }
};


inline void Context::free_pipe() {
    for (Batch* b : pipe) delete b;
    pipe.clear();
}

// Result fields from counts (FinalRule::setMeasures / setConfidence).
void compose(const RulePlan& rp, int64_t sup, int64_t body, double supMs, double confMs, GpuRuleResult* out);

}  // namespace gr
