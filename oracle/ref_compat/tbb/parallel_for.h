// Minimal stand-in for tbb::parallel_for over std::thread (reference call
// sites: sys/tasking.h:39-51, image/accum_buffer.h:109-120,266-305).
// The range is cut into one contiguous chunk per worker; worker k runs with
// current_thread_index() == k, which is what Tasking::run relies on to pick
// its per-thread state. Test infrastructure only.
#pragma once

#include <algorithm>
#include <thread>
#include <vector>
#include "blocked_range.h"
#include "task_arena.h"

namespace tbb {

struct static_partitioner {};
struct auto_partitioner {};

template <class T, class Body>
inline void parallel_for(const blocked_range<T>& range, const Body& body)
{
    const T n = range.end() - range.begin();
    if (n <= 0) return;
    int workers = std::min<long long>((long long)n, (long long)detail_shim::workerCount());
    if (workers <= 1)
    {
        detail_shim::threadIndex() = 0;
        body(range);
        return;
    }
    auto chunk = [&](int k) {
        T lo = range.begin() + (T)((long long)n * k / workers);
        T hi = range.begin() + (T)((long long)n * (k + 1) / workers);
        detail_shim::threadIndex() = k;
        if (lo < hi) body(blocked_range<T>(lo, hi));
    };
    std::vector<std::thread> pool;
    pool.reserve(workers - 1);
    for (int k = 1; k < workers; ++k)
        pool.emplace_back(chunk, k);
    chunk(0);
    for (auto& t : pool) t.join();
    detail_shim::threadIndex() = 0;
}

template <class T, class Body, class Partitioner>
inline void parallel_for(const blocked_range<T>& range, const Body& body, Partitioner)
{
    parallel_for(range, body);
}

} // namespace tbb
