// parallel.hpp — a blocking parallel loop over host threads for the batch
// preparation (parsing, planning and task building of large rule batches).
#pragma once
#include <algorithm>
#include <atomic>
#include <exception>
#include <mutex>
#include <thread>
#include <vector>

namespace gr {

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
    std::vector<std::thread> pool;
    pool.reserve(t - 1);
    for (unsigned k = 1; k < t; ++k) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
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
