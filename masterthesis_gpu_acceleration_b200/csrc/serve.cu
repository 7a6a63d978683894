// serve.cu — continuous-batching request loop on a resident graph.
//
// A server owns one worker thread and a few launch slots (each a stream with
// its own staged device buffers).  Requests (rule texts) are queued by any
// thread.  Whenever a slot is free the worker takes the waiting requests, in
// arrival order, up to a batch limit and within the device-memory budget
// (each request's estimated plan, task and dedup-buffer bytes; the rest wait
// for memory to be released), plans them and launches one persistent kernel
// for all of them on that slot's stream without waiting.  Requests that
// arrive while other launches are on the GPU go into the next free slot, so
// launches overlap on the device.  The worker retires a slot when its event
// completes and publishes each request's result with its latency from
// submission to completion.  The reference has no counterpart (it evaluates
// one rule per call, GPU_03/gpu_rules_lib.cu:330-543).
#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>

#include "engine.hpp"

namespace gr {
namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    long long id;
    std::string text;
    Clock::time_point t0;
};

struct Slot {
    Staged st;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    bool busy = false;
    size_t mem = 0;
    std::vector<Request> reqs;
    std::vector<RulePlan> rps;
    std::vector<int> parseStatus;
    std::vector<int> owner;
};

}  // namespace

struct Server {
    Context* c = nullptr;
    int maxBatch = 4096;
    size_t memBudget = 1ull << 30;
    std::vector<std::unique_ptr<Slot>> slots;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cvWork, cvDone;
    std::deque<Request> pending;
    std::deque<GpuServeResult> done;
    bool stopping = false;
    size_t memInUse = 0;
    long long submitted = 0, completed = 0, launches = 0;
    double deviceBusyMs = 0;
    std::string error;

    // Bytes a request may hold on the device while in flight.
    size_t estimate(const RulePlan& rp) const {
        size_t b = 0;
        for (const PhasePlan* ph : {&rp.support, &rp.body}) {
            if (ph->how != kDevice) continue;
            const DevPlan& P = ph->plan;
            size_t roots = (size_t)std::max(1, ph->rootEnd - ph->rootBeg);
            size_t tasks = roots / (size_t)std::max(1, std::min(P.groupMax, P.cap)) + 1;
            b += sizeof(DevPlan) + 8 + tasks * sizeof(DevTask) * 2;
            if (ph->needsGlobalBitmap) b += roots * (size_t)P.wo / 8 + 4;
        }
        return b;
    }

    void retire(Slot& s) {
        cudaError_t e = cudaEventQuery(s.done);
        if (e == cudaErrorNotReady) return;
        auto now = Clock::now();
        int status = 0;
        if (e != cudaSuccess) {
            status = -3;
            error = cudaGetErrorString(e);
            cudaGetLastError();
        } else if (s.st.nPlans && static_cast<const int*>(s.st.hCtl.p)[1] != 0) {
            status = -3;
            error = "engine reported internal status";
        }
        std::vector<int64_t> sup(s.reqs.size()), body(s.reqs.size());
        for (size_t i = 0; i < s.reqs.size(); ++i) { sup[i] = s.rps[i].support.value; body[i] = s.rps[i].body.value; }
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
            for (size_t i = 0; i < s.reqs.size(); ++i) {
                GpuServeResult r{};
                r.requestId = s.reqs[i].id;
                r.status = s.parseStatus[i] != 0 ? s.parseStatus[i] : status;
                if (r.status == 0) compose(s.rps[i], sup[i], body[i], 0.0, 0.0, &r.result);
                r.latencyMs = std::chrono::duration<double, std::milli>(now - s.reqs[i].t0).count();
                done.push_back(r);
            }
            completed += (long long)s.reqs.size();
            memInUse -= s.mem;
        }
        cvDone.notify_all();
        s.busy = false;
        s.reqs.clear();
    }

    // Takes admitted requests into a free slot and launches them.
    bool launch(Slot& s) {
        std::vector<Request> take;
        {
            std::lock_guard<std::mutex> lk(mu);
            while (!pending.empty() && (int)take.size() < maxBatch) {
                take.push_back(std::move(pending.front()));
                pending.pop_front();
            }
        }
        if (take.empty()) return false;
        s.rps.assign(take.size(), RulePlan{});
        s.parseStatus.assign(take.size(), 0);
        s.owner.clear();
        std::vector<DevPlan> plans;
        std::vector<const PhasePlan*> phases;
        size_t mem = 0;
        size_t admitted = 0;
        size_t budgetLeft;
        {
            std::lock_guard<std::mutex> lk(mu);
            budgetLeft = memBudget > memInUse ? memBudget - memInUse : 0;
        }
        size_t inUse;
        {
            std::lock_guard<std::mutex> lk(mu);
            inUse = memInUse;
        }
        std::vector<Request> back;
        for (size_t i = 0; i < take.size(); ++i) {
            RulePlan rp;
            int ps = 0;
            try {
                rp = plan_rule(c->parser->parse_text(take[i].text), c->hix, c->geom);
            } catch (const std::exception&) {
                ps = -1;
            }
            size_t m = ps ? 0 : estimate(rp);
            if (m > memBudget) { ps = -2; m = 0; }   // can never fit: rejected
            if (mem + m > budgetLeft && (admitted > 0 || inUse > 0)) {
                // no memory for it now: it waits, in order, with the rest
                back.assign(std::make_move_iterator(take.begin() + i), std::make_move_iterator(take.end()));
                break;
            }
            mem += m;
            s.rps[admitted] = std::move(rp);
            s.parseStatus[admitted] = ps;
            if (admitted != i) take[admitted] = std::move(take[i]);
            ++admitted;
        }
        take.resize(admitted);
        s.rps.resize(admitted);
        s.parseStatus.resize(admitted);
        if (!back.empty()) {
            std::lock_guard<std::mutex> lk(mu);
            for (auto it = back.rbegin(); it != back.rend(); ++it) pending.push_front(std::move(*it));
        }
        if (admitted == 0) return false;
        for (size_t i = 0; i < admitted; ++i) {
            RulePlan& rp = s.rps[i];
            if (s.parseStatus[i] != 0 || rp.status != kRuleOk) continue;
            if (rp.support.how == kDevice) { plans.push_back(rp.support.plan); phases.push_back(&rp.support); s.owner.push_back(2 * (int)i); }
            if (rp.body.how == kDevice) { plans.push_back(rp.body.plan); phases.push_back(&rp.body); s.owner.push_back(2 * (int)i + 1); }
        }
        s.reqs = std::move(take);
        s.mem = mem;
        {
            std::lock_guard<std::mutex> lk(mu);
            memInUse += mem;
        }
        s.st.stage(*c, plans, phases, true, s.stream);
        s.st.enqueue(*c, s.stream, false);
        s.st.download(s.stream);
        ck(cudaEventRecord(s.done, s.stream), "event");
        s.busy = true;
        ++launches;
        return true;
    }

    void run() {
        cudaSetDevice(c->device);
        for (;;) {
            bool any = false, busy = false;
            for (auto& s : slots)
                if (s->busy) { retire(*s); busy |= s->busy; }
            for (auto& s : slots) {
                if (s->busy) continue;
                bool has;
                {
                    std::lock_guard<std::mutex> lk(mu);
                    has = !pending.empty();
                }
                if (!has) break;
                try {
                    any |= launch(*s);
                } catch (const std::exception& e) {
                    // fail the requests of this launch, keep serving
                    std::lock_guard<std::mutex> lk(mu);
                    error = e.what();
                    for (auto& r : s->reqs) {
                        GpuServeResult x{};
                        x.requestId = r.id;
                        x.status = -3;
                        done.push_back(x);
                    }
                    completed += (long long)s->reqs.size();
                    memInUse -= s->mem;
                    s->reqs.clear();
                    s->busy = false;
                    cudaGetLastError();
                    cvDone.notify_all();
                }
                busy |= s->busy;
            }
            std::unique_lock<std::mutex> lk(mu);
            if (stopping && pending.empty() && !busy) break;
            if (!any) {
                if (busy) {
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
            if (s->done) cudaEventDestroy(s->done);
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
        ck(cudaSetDevice(sv->c->device), "cudaSetDevice");
        for (int i = 0; i < slots; ++i) {
            auto s = std::make_unique<Slot>();
            ck(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "cudaStreamCreate");
            ck(cudaEventCreateWithFlags(&s->done, cudaEventDisableTiming), "cudaEventCreate");
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
                    long long* memInUse) {
    if (!server) return -1;
    Server& sv = *static_cast<Server*>(server);
    std::lock_guard<std::mutex> lk(sv.mu);
    if (submitted) *submitted = sv.submitted;
    if (completed) *completed = sv.completed;
    if (launches) *launches = sv.launches;
    if (memInUse) *memInUse = (long long)sv.memInUse;
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
