// context.cu — graph context and the C ABI (include/gpu_rules_api.h).
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
#include <cstdio>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/gpu_rules_api.h"
#include "common.hpp"
#include "index.hpp"
#include "planner.hpp"
#include "rules.hpp"
#include "turtle.hpp"

namespace gr {

size_t engine_smem_bytes();
cudaError_t engine_configure();
cudaError_t engine_launch(const DevIndex& ix, const DevPlan* plans, const DevTask* tasks, int nTasks,
                          int* taskCounter, unsigned long long* results, int* status, int grid,
                          cudaStream_t stream);

namespace {

thread_local std::string g_lastError;

void set_error(const std::string& s) {
    g_lastError = s;
    std::fprintf(stderr, "[gpu_rules] %s\n", s.c_str());
}

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

inline void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    void ensure(size_t bytes) {
        if (bytes <= cap) return;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        size_t want = std::max<size_t>(bytes, 4096);
        ck(cudaMalloc(&p, want), "cudaMalloc");
        cap = want;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

}  // namespace

struct Context {
    int device = 0;
    TermDict ents, preds;
    std::unordered_map<std::string, std::string> prefixes;
    HostIndex hix;
    void* indexMem = nullptr;
    DevIndex dix{};
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {};
    DevBuf plans, tasks, results, ctl, gbitmap;
    int grid = 0;
    std::unique_ptr<RuleParser> parser;

    ~Context() {
        cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        plans.release(); tasks.release(); results.release(); ctl.release(); gbitmap.release();
        if (indexMem) cudaFree(indexMem);
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
        ck(cudaMalloc(&indexMem, std::max<size_t>(total, 256)), "cudaMalloc(index)");
        char* base = static_cast<char*>(indexMem);
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
        dix.hashMask = h.hashMask;
        dix.nPred = h.nPred;
        dix.nEnt = h.nEnt;
        dix.nTriples = h.nTriples;
    }

    void init_device() {
        ck(cudaGetDevice(&device), "cudaGetDevice");
        int sms = 0;
        ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "cudaDeviceGetAttribute");
        ck(engine_configure(), "cudaFuncSetAttribute");
        grid = sms * 2;
        ck(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
        for (auto& e : ev) ck(cudaEventCreate(&e), "cudaEventCreate");
        ctl.ensure(256);
    }

    int* counter() { return static_cast<int*>(ctl.p); }
    int* status() { return static_cast<int*>(ctl.p) + 1; }
};

namespace {

struct PhaseRun {
    const PhasePlan* ph;
    DevPlan plan;
};

int64_t clamp_int(int64_t v) { return std::min<int64_t>(v, INT_MAX); }

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

// Runs the given phases (one plan each) in one launch; results[i] receives
// plan i's count.  Global bitmaps are carved from the context's arena.
void run_phases(Context& c, std::vector<DevPlan>& plans, const std::vector<const PhasePlan*>& phases,
                std::vector<unsigned long long>& counts, float* ms, bool sortTasks) {
    size_t n = plans.size();
    counts.assign(n, 0);
    if (ms) *ms = 0.f;
    if (!n) return;
    // global bitmaps
    size_t gWords = 0;
    std::vector<size_t> gOff(n, 0);
    for (size_t i = 0; i < n; ++i) {
        if (!phases[i]->needsGlobalBitmap) continue;
        size_t rows = (size_t)(phases[i]->rootEnd - phases[i]->rootBeg);
        gOff[i] = gWords;
        gWords += (rows * (size_t)plans[i].wo + 31) / 32;
    }
    if (gWords) {
        c.gbitmap.ensure(gWords * 4);
        ck(cudaMemsetAsync(c.gbitmap.p, 0, gWords * 4, c.stream), "cudaMemsetAsync(bitmap)");
    }
    std::vector<DevTask> tasks;
    std::vector<double> cost;
    for (size_t i = 0; i < n; ++i) {
        plans[i].resultSlot = (int32_t)i;
        if (phases[i]->needsGlobalBitmap) {
            plans[i].gBitmap = static_cast<uint32_t*>(c.gbitmap.p) + gOff[i];
            plans[i].gRowBase = phases[i]->rootBeg;
        } else {
            plans[i].gBitmap = nullptr;
        }
        make_tasks(*phases[i], (int32_t)i, c.hix, tasks, &cost);
    }
    if (sortTasks && tasks.size() > 1) {
        std::vector<size_t> ord(tasks.size());
        std::iota(ord.begin(), ord.end(), 0);
        std::stable_sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return cost[a] > cost[b]; });
        std::vector<DevTask> t2(tasks.size());
        for (size_t i = 0; i < ord.size(); ++i) t2[i] = tasks[ord[i]];
        tasks.swap(t2);
    }
    c.plans.ensure(n * sizeof(DevPlan));
    c.tasks.ensure(std::max<size_t>(tasks.size(), 1) * sizeof(DevTask));
    c.results.ensure(n * sizeof(unsigned long long));
    ck(cudaMemcpyAsync(c.plans.p, plans.data(), n * sizeof(DevPlan), cudaMemcpyHostToDevice, c.stream), "H2D plans");
    if (!tasks.empty())
        ck(cudaMemcpyAsync(c.tasks.p, tasks.data(), tasks.size() * sizeof(DevTask), cudaMemcpyHostToDevice, c.stream), "H2D tasks");
    ck(cudaMemsetAsync(c.results.p, 0, n * sizeof(unsigned long long), c.stream), "memset results");
    ck(cudaMemsetAsync(c.ctl.p, 0, 8, c.stream), "memset ctl");
    ck(cudaEventRecord(c.ev[0], c.stream), "event");
    int grid = std::min<int>((int)tasks.size(), c.grid);
    ck(engine_launch(c.dix, static_cast<const DevPlan*>(c.plans.p), static_cast<const DevTask*>(c.tasks.p),
                     (int)tasks.size(), c.counter(), static_cast<unsigned long long*>(c.results.p), c.status(),
                     std::max(grid, 1), c.stream), "engine launch");
    ck(cudaEventRecord(c.ev[1], c.stream), "event");
    int st[2] = {0, 0};
    ck(cudaMemcpyAsync(counts.data(), c.results.p, n * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c.stream), "D2H results");
    ck(cudaMemcpyAsync(st, c.ctl.p, 8, cudaMemcpyDeviceToHost, c.stream), "D2H status");
    ck(cudaStreamSynchronize(c.stream), "kernel");
    if (ms) ck(cudaEventElapsedTime(ms, c.ev[0], c.ev[1]), "elapsed");
    if (st[1] != 0) throw CudaError("engine reported internal status " + std::to_string(st[1]));
}

int evaluate_parsed(Context& c, const Rule& rule, GpuRuleResult* out) {
    RulePlan rp = plan_rule(rule, c.hix);
    int64_t sup = rp.support.value, body = rp.body.value;
    float supMs = 0.f, confMs = 0.f;
    std::vector<unsigned long long> counts;
    if (rp.status == kRuleOk && rp.support.how == kDevice) {
        std::vector<DevPlan> plans{rp.support.plan};
        run_phases(c, plans, {&rp.support}, counts, &supMs, false);
        sup = (int64_t)counts[0];
    }
    if (rp.status == kRuleOk && rp.body.how == kDevice) {
        std::vector<DevPlan> plans{rp.body.plan};
        run_phases(c, plans, {&rp.body}, counts, &confMs, false);
        body = (int64_t)counts[0];
    }
    compose(rp, sup, body, supMs, confMs, out);
    return 0;
}

Context* as_ctx(void* p) { return static_cast<Context*>(p); }

}  // namespace
}  // namespace gr

using namespace gr;

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
        std::string err;
        if (!parse_turtle_file(ttlPath, c->ents, c->preds, spo, &err)) {
            set_error("Failed to parse TTL: " + std::string(ttlPath) + " (" + err + ")");
            delete c;
            return nullptr;
        }
        c->prefixes = scan_rule_prefixes(ttlPath);
        c->hix = build_index(spo, (int32_t)c->ents.size(), (int32_t)c->preds.size());
        c->parser.reset(new RuleParser(c->ents, c->preds, c->prefixes));
        c->init_device();
        c->upload_index();
        return c;
    } catch (const std::exception& e) {
        set_error(std::string("gpu_load_graph error: ") + e.what());
        cudaGetLastError();
        delete c;
        return nullptr;
    }
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
    if (!ctx || (!rules && n > 0) || (!out && n > 0) || n < 0) return -1;
    Context& c = *as_ctx(ctx);
    if (deviceMs) *deviceMs = 0.0;
    try {
        cudaSetDevice(c.device);
        std::vector<RulePlan> rps(n);
        std::vector<DevPlan> plans;
        std::vector<const PhasePlan*> phases;
        std::vector<int> owner;  // plan -> rule*2 + phase
        plans.reserve(2 * (size_t)n);
        for (int i = 0; i < n; ++i) {
            out[i] = GpuRuleResult{};
            if (status) status[i] = 0;
            if (!rules[i]) { if (status) status[i] = -1; rps[i].status = -1; continue; }
            try {
                Rule r = isJson ? c.parser->parse_json(rules[i]) : c.parser->parse_text(rules[i]);
                rps[i] = plan_rule(r, c.hix);
            } catch (const RuleError& e) {
                if (status) status[i] = -1;
                rps[i].status = -1;
                continue;
            }
            if (rps[i].status != kRuleOk) continue;
            if (rps[i].support.how == kDevice) {
                plans.push_back(rps[i].support.plan);
                phases.push_back(&rps[i].support);
                owner.push_back(2 * i);
            }
            if (rps[i].body.how == kDevice) {
                plans.push_back(rps[i].body.plan);
                phases.push_back(&rps[i].body);
                owner.push_back(2 * i + 1);
            }
        }
        std::vector<unsigned long long> counts;
        float ms = 0.f;
        run_phases(c, plans, phases, counts, &ms, true);
        std::vector<int64_t> sup(n), body(n);
        for (int i = 0; i < n; ++i) { sup[i] = rps[i].support.value; body[i] = rps[i].body.value; }
        for (size_t k = 0; k < owner.size(); ++k) {
            int i = owner[k] / 2;
            if (owner[k] % 2 == 0) sup[i] = (int64_t)counts[k];
            else body[i] = (int64_t)counts[k];
        }
        for (int i = 0; i < n; ++i) {
            if (rps[i].status == -1) continue;
            compose(rps[i], sup[i], body[i], 0.0, 0.0, &out[i]);
        }
        if (deviceMs) *deviceMs = ms;
        return 0;
    } catch (const std::exception& e) {
        set_error(std::string("gpu_evaluate_rules_batch error: ") + e.what());
        return -1;
    }
}

int gpu_graph_stats(void* ctx, long long* entities, long long* predicates, long long* triples) {
    if (!ctx) return -1;
    Context& c = *as_ctx(ctx);
    if (entities) *entities = (long long)c.hix.nEnt;
    if (predicates) *predicates = (long long)c.hix.nPred;
    if (triples) *triples = (long long)c.hix.nTriples;
    return 0;
}

}  // extern "C"
