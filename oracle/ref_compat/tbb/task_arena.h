// Minimal stand-in for tbb::this_task_arena (reference: sys/tasking.h:54-62).
// The worker count comes from PRT_REF_THREADS when set, else from the number
// of online cores; it never exceeds the configured core count, because the
// reference sizes its per-thread state arrays with sysconf(_SC_NPROCESSORS_CONF)
// (sys/sysinfo.cpp:34,50-61). Test infrastructure only.
#pragma once

#include <cstdlib>
#include <thread>
#include <unistd.h>

namespace tbb {
namespace detail_shim {

inline int& threadIndex()
{
    static thread_local int index = 0;
    return index;
}

inline int workerCount()
{
    static int n = [] {
        int conf = (int)sysconf(_SC_NPROCESSORS_CONF);
        int online = (int)std::thread::hardware_concurrency();
        int count = online > 0 ? online : 1;
        if (const char* env = std::getenv("PRT_REF_THREADS"))
        {
            int req = std::atoi(env);
            if (req > 0) count = req;
        }
        if (conf > 0 && count > conf) count = conf;
        return count;
    }();
    return n;
}

} // namespace detail_shim

namespace this_task_arena {
inline int max_concurrency() { return detail_shim::workerCount(); }
inline int current_thread_index() { return detail_shim::threadIndex(); }
} // namespace this_task_arena

} // namespace tbb
