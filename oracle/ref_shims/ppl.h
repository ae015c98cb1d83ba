/* Linux stand-in for the MSVC Parallel Patterns Library header used by the
 * reference's BVHCPUBuilder (minimum_lbvh.h:22, :565). parallel_for splits
 * [first, last) into contiguous chunks over std::thread workers.
 * Test infrastructure only (oracle/_ref). */
#pragma once
#include <thread>
#include <vector>
#include <algorithm>
#include <cstdlib>

namespace concurrency
{
    inline unsigned oracle_thread_count()
    {
        const char* env = std::getenv("MLBVH_ORACLE_THREADS");
        if (env && std::atoi(env) > 0) return (unsigned)std::atoi(env);
        unsigned n = std::thread::hardware_concurrency();
        return n ? n : 1;
    }

    template <class Index, class Func>
    void parallel_for(Index first, Index last, const Func& f)
    {
        if (!(first < last)) return;
        size_t total = (size_t)(last - first);
        unsigned nthreads = (unsigned)std::min<size_t>(oracle_thread_count(), total);
        if (nthreads <= 1)
        {
            for (Index i = first; i < last; ++i) f(i);
            return;
        }
        std::vector<std::thread> workers;
        size_t chunk = (total + nthreads - 1) / nthreads;
        for (unsigned t = 0; t < nthreads; ++t)
        {
            size_t b = t * chunk, e = std::min(total, b + chunk);
            if (b >= e) break;
            workers.emplace_back([=, &f]() {
                for (size_t i = b; i < e; ++i) f((Index)(first + (Index)i));
            });
        }
        for (auto& w : workers) w.join();
    }
}
