// parallel.hpp — a blocking parallel loop over host threads for the batch
// preparation (parsing, planning and task building of large rule batches).
#pragma once
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <exception>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace gr {

// Worker threads started once per process and reused by every parallel
// loop: starting threads per loop cost about as much as the preparation of
// a batch chunk itself.  One loop runs on the pool at a time; a loop that
// finds it busy with another host thread's loop starts threads of its own,
// and a loop nested in a pool loop's body, or in a process forked after the
// pool started, runs on its calling thread alone.
class HostPool {
public:
    // Never destroyed: its workers end with the process (a forked child,
    // which has none of them, must not wait for them either).
    static HostPool& get() {
        static HostPool* pool = new HostPool();
        return *pool;
    }
    // Runs work() on the calling thread and on up to n - 1 workers and
    // returns when all have returned; false (nothing run) when the pool is
    // busy or belongs to another process.
    bool run(unsigned n, const std::function<void()>& work) {
        if (inWorker() || inRegion() || ::getpid() != pid_) return false;
        std::unique_lock<std::mutex> region(regionMu_, std::try_to_lock);
        if (!region.owns_lock()) return false;
        struct Mark {   // loops nested in this one's body, on this thread, do not touch the lock
            Mark() { inRegion() = true; }
            ~Mark() { inRegion() = false; }
        } mark;
        const unsigned helpers = std::min<unsigned>(n > 0 ? n - 1 : 0, nWorkers_);
        job_ = &work;
        pending_.store(helpers, std::memory_order_relaxed);
        {
            // generation and helper count in one word: a worker that sees a
            // generation late reads the count of that same generation
            std::lock_guard<std::mutex> lk(mu_);   // a sleeping worker sees the new generation
            const uint64_t g = (ctl_.load(std::memory_order_relaxed) >> 8) + 1;
            ctl_.store((g << 8) | helpers, std::memory_order_release);
        }
        cv_.notify_all();
        work();
        while (pending_.load(std::memory_order_acquire) != 0) std::this_thread::yield();
        job_ = nullptr;
        return true;
    }
    // Whether this process started the pool (not a forked child).
    bool own_process() const { return ::getpid() == pid_; }
    // Whether the calling thread is one of the pool's workers, or runs a
    // pool loop's body on the calling side.
    static bool in_worker() { return inWorker() || inRegion(); }

private:
    HostPool() : pid_(::getpid()) {
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        for (unsigned i = 0; i + 1 < std::min(hw, 64u); ++i) std::thread([this, i] { loop(i); }).detach();
        nWorkers_ = std::max(1u, std::min(hw, 64u)) - 1;
    }
    static bool& inWorker() {
        static thread_local bool w = false;
        return w;
    }
    static bool& inRegion() {
        static thread_local bool r = false;
        return r;
    }
    // After each loop a worker polls for the next one for a while (the
    // loops of one batch come a few hundred microseconds apart), then
    // sleeps until woken.
    void loop(unsigned idx) {
        inWorker() = true;
        uint64_t seen = 0;   // the generation when the pool started (a loop may come before this thread runs)
        for (;;) {
            uint64_t c = ctl_.load(std::memory_order_acquire);
            for (int spin = 0; (c >> 8) == seen && spin < 4000; ++spin) {
                std::this_thread::yield();
                c = ctl_.load(std::memory_order_acquire);
            }
            if ((c >> 8) == seen) {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return (ctl_.load(std::memory_order_acquire) >> 8) != seen; });
                c = ctl_.load(std::memory_order_acquire);
            }
            seen = c >> 8;
            // a helper of this generation: the caller waits for it, so job_
            // still holds this generation's loop
            if (idx >= (unsigned)(c & 0xffu)) continue;
            (*job_)();
            pending_.fetch_sub(1, std::memory_order_acq_rel);
        }
    }
    unsigned nWorkers_ = 0;
    std::mutex mu_, regionMu_;
    std::condition_variable cv_;
    const std::function<void()>* job_ = nullptr;   // written before ctl_ is raised
    std::atomic<unsigned> pending_{0};
    std::atomic<uint64_t> ctl_{0};   // generation << 8 | helpers wanted (at most 63)
    const pid_t pid_;
};

// Calls fn(i) for i in [0, n) on up to maxThreads threads (the calling
// thread included), in chunks of `grain`; serial below 2 * grain items.
// The first exception thrown by fn stops the loop and is rethrown here.
template <class Fn>
void parallel_for(size_t n, Fn fn, size_t grain = 64, unsigned maxThreads = 16) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned t = (unsigned)std::min<size_t>(std::min(hw, maxThreads), n / std::max<size_t>(grain, 1));
    if (t <= 1) {
        for (size_t i = 0; i < n; ++i) fn(i);
        return;
    }
    std::atomic<size_t> next{0};
    std::exception_ptr err;
    std::mutex errMu;
    auto work = [&] {
        try {
            for (;;) {
                const size_t b = next.fetch_add(grain);
                if (b >= n) return;
                const size_t e = std::min(n, b + grain);
                for (size_t i = b; i < e; ++i) fn(i);
            }
        } catch (...) {
            std::lock_guard<std::mutex> lk(errMu);
            if (!err) err = std::current_exception();
            next = n;
        }
    };
    const std::function<void()> job(work);
    if (!HostPool::get().run(t, job)) {
        if (HostPool::in_worker() || !HostPool::get().own_process()) {
            work();   // nested in a pool loop's body: the pool's threads are busy with it
        } else {
            // the pool runs another host thread's loop (two servers planning
            // at once, say): this loop starts threads of its own
            std::vector<std::thread> extra;
            extra.reserve(t - 1);
            for (unsigned k = 1; k < t; ++k) extra.emplace_back(work);
            work();
            for (auto& th : extra) th.join();
        }
    }
    if (err) std::rethrow_exception(err);
}

// Sorts v with cmp on several threads: chunks are sorted in parallel, then
// merged pairwise, level by level, in parallel.
template <class T, class Cmp>
void parallel_sort(std::vector<T>& v, Cmp cmp, size_t minChunk = size_t(1) << 16) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    size_t parts = std::min<size_t>(std::min(hw, 16u), v.size() / std::max<size_t>(minChunk, 1));
    if (parts < 2) {
        std::sort(v.begin(), v.end(), cmp);
        return;
    }
    std::vector<size_t> b(parts + 1);
    for (size_t k = 0; k <= parts; ++k) b[k] = v.size() * k / parts;
    parallel_for(parts, [&](size_t k) { std::sort(v.begin() + b[k], v.begin() + b[k + 1], cmp); }, 1);
    for (size_t width = 1; width < parts; width *= 2) {
        const size_t pairs = (parts + 2 * width - 1) / (2 * width);
        parallel_for(pairs, [&](size_t q) {
            const size_t lo = 2 * width * q, mid = std::min(parts, lo + width), hi = std::min(parts, lo + 2 * width);
            if (mid < hi) std::inplace_merge(v.begin() + b[lo], v.begin() + b[mid], v.begin() + b[hi], cmp);
        }, 1);
    }
}

}  // namespace gr
