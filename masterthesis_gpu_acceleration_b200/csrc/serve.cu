// serve.cu — continuous-batching request loop on a resident graph.
//
// A server owns one worker thread and a few launch slots (each a stream with
// its own pre-sized device buffers).  Requests (rule texts) are queued by any
// thread.  The worker parses and plans them as they arrive and sorts them
// into two lanes by their expected device time: light requests, and heavy
// ones (long chains through hub entities, whose enumeration can take far
// longer than the rest).  Whenever a light slot is free the worker launches
// every waiting light request, in arrival order, up to a batch limit and
// within the device-memory budget (each request's estimated plan, task and
// dedup-buffer bytes; the rest wait for memory to be released), as one
// persistent kernel on that slot's stream without waiting for it.  Heavy
// requests go to their own slot, launched on half of the SMs, so that
// they never hold the whole GPU while light requests queue behind them.
// When heavy work piles up (more expected device time waiting than a few
// heavy batches) and no light request waits, light slots take heavy
// requests too, so that an overloaded server keeps every slot busy.
// Requests arriving while launches run are batched into the next free slot,
// so launches overlap on the device.  A slot is retired when its event
// completes; each request's result is published with its latency from
// submission to completion.  The reference has no counterpart (it evaluates
// one rule per call, GPU_03/gpu_rules_lib.cu:330-543).
#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>

#include "engine.hpp"
#include "parallel.hpp"

namespace gr {
namespace {

using Clock = std::chrono::steady_clock;

constexpr size_t kReservePlans = 16384;  // launch sizes that never resize a slot's buffers
constexpr size_t kReserveTasks = 1 << 18;
constexpr double kOverflowBatches = 4;   // heavy backlog, in heavy thresholds, that opens overflow
constexpr double kWalkAfterNs = 1.0e6;   // a plan whose slowest task took longer is walked next time

struct Request {
    long long id;
    std::string text;
    Clock::time_point t0;
};

struct Planned {
    Request req;
    RulePlan rp;
    int status = 0;   // 0, or -1 (parse) / -2 (too large)
    size_t mem = 0;
    double ns = 0;    // expected device time
};

struct Slot {
    Staged st;
    bool heavyLane = false;
    cudaStream_t stream = nullptr;
    cudaEvent_t start = nullptr, kend = nullptr, done = nullptr;   // done: results are on the host
    bool busy = false;
    bool timed = false;                        // task times are recorded for learning
    int grid = 0;
    size_t mem = 0;
    std::vector<Planned> reqs;
    std::vector<int> owner;
    std::vector<const PhasePlan*> phases;
    HostBuf hTaskNs;
};

}  // namespace

struct Server {
    Context* c = nullptr;
    int maxBatch = 4096;
    size_t memBudget = 1ull << 30;
    bool lanes = true;                      // a separate heavy lane (two or more slots)
    std::vector<std::unique_ptr<Slot>> slots;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cvWork, cvDone;
    std::deque<Request> pending;            // submitted, not yet planned (shared)
    std::deque<Planned> light, heavy;       // planned, waiting for a slot (worker only)
    double heavyBacklogNs = 0;              // expected device time in `heavy`
    std::deque<GpuServeResult> done;
    bool stopping = false;
    size_t memInUse = 0;
    long long submitted = 0, completed = 0, launches = 0;
    double deviceMs = 0, hostMs = 0;        // summed launch spans, host preparation time
    std::string error;

    // Bytes a request may hold on the device while in flight.
    size_t estimate_mem(const RulePlan& rp) const {
        size_t b = 0;
        for (const PhasePlan* ph : {&rp.support, &rp.body}) {
            if (ph->how != kDevice) continue;
            const DevPlan& P = ph->plan;
            size_t roots = (size_t)std::max(1, ph->rootEnd - ph->rootBeg);
            size_t tasks = roots / (size_t)std::max(1, std::min(P.groupMax, P.cap)) + 1;
            b += sizeof(DevPlan) + 8 + tasks * sizeof(DevTask) * 2;
            if (ph->needsGlobalBitmap) b += std::min(roots * (size_t)std::max(P.rowWords, 1) * 4, c->dedupBudget);
        }
        return b;
    }

    void publish(const Planned& q, int status, int64_t sup, int64_t body, Clock::time_point now) {
        GpuServeResult r{};
        r.requestId = q.req.id;
        r.status = q.status != 0 ? q.status : status;
        if (r.status == 0) compose(q.rp, sup, body, 0.0, 0.0, &r.result);
        r.latencyMs = std::chrono::duration<double, std::milli>(now - q.req.t0).count();
        done.push_back(r);
    }

    void retire(Slot& s) {
        cudaError_t e = cudaEventQuery(s.done);
        if (e == cudaErrorNotReady) return;
        auto now = Clock::now();
        int status = 0;
        float span = 0.f;
        if (e == cudaSuccess && cudaEventElapsedTime(&span, s.start, s.kend) == cudaSuccess) deviceMs += span;
        if (e != cudaSuccess) {
            status = -3;
            error = cudaGetErrorString(e);
            cudaGetLastError();
        } else if (s.st.nPlans && static_cast<const int*>(s.st.hCtl.p)[1] != 0) {
            status = -3;
            error = "engine reported internal status";
        }
        std::vector<int64_t> sup(s.reqs.size()), body(s.reqs.size());
        for (size_t i = 0; i < s.reqs.size(); ++i) {
            sup[i] = s.reqs[i].rp.support.value;
            body[i] = s.reqs[i].rp.body.value;
        }
        // requests that lost device work at the launch's deadline
        std::vector<char> late(s.reqs.size(), 0);
        bool anyLate = false;
        if (status == 0)
            for (size_t k = 0; k < s.owner.size(); ++k)
                if (s.st.plan_incomplete((int)k)) {
                    late[(size_t)s.owner[k] / 2] = 1;
                    anyLate = true;
                }
        if (status == 0 && s.timed && !anyLate) {   // abandoned tasks have no times to learn from
            const auto h0 = Clock::now();
            c->tasks->learn(s.phases, s.st.hTasks, s.st.hCost,
                            static_cast<const unsigned long long*>(s.hTaskNs.p), s.grid, 0.5, kWalkAfterNs);
            hostMs += std::chrono::duration<double, std::milli>(Clock::now() - h0).count();
        }
        if (status == 0) {
            const unsigned long long* cnt = s.st.counts();
            for (size_t k = 0; k < s.owner.size(); ++k) {
                size_t i = s.owner[k] / 2;
                if (s.owner[k] % 2 == 0) sup[i] = (int64_t)cnt[k];
                else body[i] = (int64_t)cnt[k];
            }
        }
        {
            std::lock_guard<std::mutex> lk(mu);
            for (size_t i = 0; i < s.reqs.size(); ++i) publish(s.reqs[i], late[i] ? -4 : status, sup[i], body[i], now);
            completed += (long long)s.reqs.size();
            memInUse -= s.mem;
        }
        cvDone.notify_all();
        s.busy = false;
        s.reqs.clear();
    }

    // Parses and plans newly submitted requests into the two lanes.
    bool plan_pending() {
        std::deque<Request> got;
        {
            std::lock_guard<std::mutex> lk(mu);
            got.swap(pending);
        }
        if (got.empty()) return false;
        const auto h0 = Clock::now();
        // parse, plan and cost the new requests on host threads (they only
        // read the graph, the dictionaries and the learnt costs, which only
        // this thread changes, between batches)
        std::vector<Planned> qs(got.size());
        parallel_for(got.size(), [&](size_t i) {
            Planned& q = qs[i];
            q.req = std::move(got[i]);
            try {
                q.rp = plan_rule(c->parser->parse_text(q.req.text), c->hix, c->geom);
            } catch (const std::exception&) {
                q.status = -1;
            }
            double ns = 0;
            if (q.status == 0) {
                q.mem = estimate_mem(q.rp);
                if (q.mem > memBudget) { q.status = -2; q.mem = 0; }
                if (q.rp.status == kRuleOk)
                    ns = c->tasks->expected_ns(q.rp.support) + c->tasks->expected_ns(q.rp.body);
                // refused without a launch: expected to take longer than the limit
                if (q.status == 0 && c->serveMaxNs > 0 && ns > c->serveMaxNs) { q.status = -4; q.mem = 0; ns = 0; }
            }
            q.ns = ns;
        }, 64);
        for (Planned& q : qs) {
            const double ns = q.ns;
            if (lanes && ns > c->serveHeavyNs) {
                heavyBacklogNs += ns;
                heavy.push_back(std::move(q));
            } else {
                light.push_back(std::move(q));
            }
        }
        hostMs += std::chrono::duration<double, std::milli>(Clock::now() - h0).count();
        return true;
    }

    // Launches the waiting requests of the slot's lane that fit the memory budget.
    bool launch(Slot& s) {
        // A light slot overflows into the heavy lane once the heavy backlog
        // exceeds what the heavy slot clears in a few batches.
        const bool overflow = !s.heavyLane && light.empty() &&
                              heavyBacklogNs > kOverflowBatches * c->serveHeavyNs;
        std::deque<Planned>& q = (s.heavyLane || overflow) ? heavy : light;
        if (q.empty()) return false;
        const auto h0 = Clock::now();
        size_t inUse;
        {
            std::lock_guard<std::mutex> lk(mu);
            inUse = memInUse;
        }
        const size_t left = memBudget > inUse ? memBudget - inUse : 0;
        size_t mem = 0;
        s.reqs.clear();
        while (!q.empty() && (int)s.reqs.size() < maxBatch) {
            const size_t m = q.front().mem;
            if (mem + m > left && (!s.reqs.empty() || inUse > 0)) break;   // waits for memory, in order
            mem += m;
            if (&q == &heavy) heavyBacklogNs = std::max(0.0, heavyBacklogNs - q.front().ns);
            s.reqs.push_back(std::move(q.front()));
            q.pop_front();
        }
        if (s.reqs.empty()) return false;
        std::vector<DevPlan> plans;
        std::vector<const PhasePlan*> phases;
        s.owner.clear();
        for (size_t i = 0; i < s.reqs.size(); ++i) {
            RulePlan& rp = s.reqs[i].rp;
            if (s.reqs[i].status != 0 || rp.status != kRuleOk) continue;
            if (rp.support.how == kDevice) { plans.push_back(rp.support.plan); phases.push_back(&rp.support); s.owner.push_back(2 * (int)i); }
            if (rp.body.how == kDevice) { plans.push_back(rp.body.plan); phases.push_back(&rp.body); s.owner.push_back(2 * (int)i + 1); }
        }
        s.mem = mem;
        {
            std::lock_guard<std::mutex> lk(mu);
            memInUse += mem;
        }
        s.busy = true;
        const bool heavyWork = s.heavyLane || overflow;
        // no sort mode: a served launch is never run a second time
        s.st.stage(*c, plans, phases, true, s.stream, heavyWork ? 4.0e6 : 2.0e5, false, false);
        // Launches record task times, from which the task builder learns
        // each plan shape's cost (the launches that follow split slow plans
        // finer and classify requests by it).
        s.timed = s.st.nTasks > 0;
        s.grid = s.heavyLane ? std::max(1, c->grid / c->serveHeavyShare) : c->grid;
        s.phases = phases;
        ck(cudaEventRecord(s.start, s.stream), "event");
        s.st.enqueue(*c, s.stream, s.timed ? 1 : 0, s.heavyLane ? s.grid : 0,
                     s.timed ? (unsigned long long)c->serveDeadlineNs : 0ull);
        ck(cudaEventRecord(s.kend, s.stream), "event");
        s.st.download(s.stream);
        if (s.timed) {
            s.hTaskNs.ensure((size_t)s.st.nTasks * 16);
            ck(cudaMemcpyAsync(s.hTaskNs.p, s.st.dTaskNs.p, (size_t)s.st.nTasks * 16, cudaMemcpyDeviceToHost,
                               s.stream),
               "D2H task times");
        }
        ck(cudaEventRecord(s.done, s.stream), "event");
        ++launches;
        hostMs += std::chrono::duration<double, std::milli>(Clock::now() - h0).count();
        return true;
    }

    void fail_slot(Slot& s, const char* what) {
        std::lock_guard<std::mutex> lk(mu);
        error = what;
        auto now = Clock::now();
        for (auto& r : s.reqs) publish(r, -3, 0, 0, now);
        completed += (long long)s.reqs.size();
        memInUse -= s.mem;
        s.reqs.clear();
        s.busy = false;
        cudaGetLastError();
        cvDone.notify_all();
    }

    void run() {
        cudaSetDevice(c->device);
        for (;;) {
            bool any = false, busy = false;
            for (auto& s : slots)
                if (s->busy) retire(*s);
            any |= plan_pending();
            for (auto& s : slots) {
                if (!s->busy) {
                    try {
                        any |= launch(*s);
                    } catch (const std::exception& e) {
                        fail_slot(*s, e.what());
                    }
                }
                busy |= s->busy;
            }
            std::unique_lock<std::mutex> lk(mu);
            if (stopping && pending.empty() && light.empty() && heavy.empty() && !busy) break;
            if (!any) {
                if (busy || !light.empty() || !heavy.empty()) {
                    lk.unlock();
                    std::this_thread::sleep_for(std::chrono::microseconds(20));
                } else {
                    cvWork.wait_for(lk, std::chrono::milliseconds(5));
                }
            }
        }
    }

    ~Server() {
        cudaSetDevice(c->device);
        for (auto& s : slots) {
            if (s->stream) cudaStreamSynchronize(s->stream);
            for (cudaEvent_t ev : {s->start, s->kend, s->done})
                if (ev) cudaEventDestroy(ev);
            if (s->stream) cudaStreamDestroy(s->stream);
        }
    }
};

}  // namespace gr

using namespace gr;

extern "C" {

void* gpu_serve_start(void* ctx, int slots, int maxBatch, long long memBudgetBytes) {
    if (!ctx || slots < 1 || slots > 16 || maxBatch < 1 || memBudgetBytes <= 0) return nullptr;
    Server* sv = nullptr;
    try {
        sv = new Server();
        sv->c = static_cast<Context*>(ctx);
        sv->maxBatch = maxBatch;
        sv->memBudget = (size_t)memBudgetBytes;
        sv->lanes = slots >= 2 && sv->c->serveLanes;   // the last slot serves the heavy lane
        ck(cudaSetDevice(sv->c->device), "cudaSetDevice");
        for (int i = 0; i < slots; ++i) {
            auto s = std::make_unique<Slot>();
            s->heavyLane = sv->lanes && i == slots - 1;
            ck(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "cudaStreamCreate");
            for (cudaEvent_t* ev : {&s->start, &s->kend, &s->done}) ck(cudaEventCreate(ev), "cudaEventCreate");
            s->st.streamOrdered = true;
            s->st.reserve(std::min<size_t>(kReservePlans, 2 * (size_t)maxBatch), kReserveTasks, s->stream);
            s->hTaskNs.ensure(kReserveTasks * 16);
            sv->slots.push_back(std::move(s));
        }
        sv->worker = std::thread([sv] { sv->run(); });
        return sv;
    } catch (const std::exception& e) {
        set_error(std::string("gpu_serve_start error: ") + e.what());
        delete sv;
        return nullptr;
    }
}

int gpu_serve_submit(void* server, long long requestId, const char* ruleText) {
    if (!server || !ruleText) return -1;
    Server& sv = *static_cast<Server*>(server);
    {
        std::lock_guard<std::mutex> lk(sv.mu);
        if (sv.stopping) return -1;
        sv.pending.push_back(Request{requestId, ruleText, Clock::now()});
        sv.submitted++;
    }
    sv.cvWork.notify_one();
    return 0;
}

int gpu_serve_poll(void* server, GpuServeResult* out, int max, int waitMs) {
    if (!server || !out || max < 0) return -1;
    Server& sv = *static_cast<Server*>(server);
    std::unique_lock<std::mutex> lk(sv.mu);
    if (sv.done.empty() && waitMs > 0)
        sv.cvDone.wait_for(lk, std::chrono::milliseconds(waitMs), [&] { return !sv.done.empty(); });
    int n = 0;
    while (n < max && !sv.done.empty()) {
        out[n++] = sv.done.front();
        sv.done.pop_front();
    }
    return n;
}

int gpu_serve_stats(void* server, long long* submitted, long long* completed, long long* launches,
                    long long* memInUse, double* deviceMs, double* hostMs) {
    if (!server) return -1;
    Server& sv = *static_cast<Server*>(server);
    std::lock_guard<std::mutex> lk(sv.mu);
    if (submitted) *submitted = sv.submitted;
    if (completed) *completed = sv.completed;
    if (launches) *launches = sv.launches;
    if (memInUse) *memInUse = (long long)sv.memInUse;
    if (deviceMs) *deviceMs = sv.deviceMs;
    if (hostMs) *hostMs = sv.hostMs;
    return 0;
}

void gpu_serve_stop(void* server) {
    if (!server) return;
    Server* sv = static_cast<Server*>(server);
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stopping = true;
    }
    sv->cvWork.notify_all();
    if (sv->worker.joinable()) sv->worker.join();
    delete sv;
}

}  // extern "C"
