// Minimal stand-in for oneTBB's parallel_for (TEST INFRASTRUCTURE); see tbb/blocked_range.h.
//
// The range is split (with its own splitting constructor and is_divisible) into at most 16 pieces
// per worker, and the pieces run on std::threads that take them in order from a shared counter. A
// parallel_for called from inside a running body (the HDK tree build nests them) runs serially in
// the calling thread. The worker count is tbb_shim::threads(), settable by the caller.
#pragma once

#include "blocked_range.h"

#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

namespace tbb {

class simple_partitioner {};
class auto_partitioner {};

} // namespace tbb

namespace tbb_shim {

inline std::atomic<int> &thread_setting() {
    static std::atomic<int> n{0};
    return n;
}
inline int threads() {
    int const n = thread_setting().load();
    return n > 0 ? n : std::max(1, static_cast<int>(std::thread::hardware_concurrency()));
}
inline void set_threads(int n) { thread_setting().store(n); }
inline bool &inside() {
    thread_local bool flag = false;
    return flag;
}

template <class Range, class Body> void run(Range const &range, Body const &body) {
    if (range.empty())
        return;
    int const workers = threads();
    if (inside() || workers == 1) {
        body(range);
        return;
    }
    std::vector<Range> pieces{range};
    std::size_t const target = static_cast<std::size_t>(workers) * 16;
    while (pieces.size() < target) {
        bool any = false;
        std::vector<Range> next;
        next.reserve(pieces.size() * 2);
        for (auto &p : pieces) {
            if (p.is_divisible()) {
                Range upper(p, tbb::split{});
                next.push_back(p);
                next.push_back(upper);
                any = true;
            } else {
                next.push_back(p);
            }
        }
        pieces.swap(next);
        if (!any)
            break;
    }
    std::atomic<std::size_t> next_piece{0};
    auto work = [&]() {
        inside() = true;
        for (std::size_t i = next_piece++; i < pieces.size(); i = next_piece++)
            body(pieces[i]);
        inside() = false;
    };
    std::vector<std::thread> pool;
    int const extra = std::min<int>(workers, static_cast<int>(pieces.size())) - 1;
    for (int t = 0; t < extra; ++t)
        pool.emplace_back(work);
    work();
    for (auto &t : pool)
        t.join();
}

} // namespace tbb_shim

namespace tbb {

template <class Range, class Body> void parallel_for(Range const &range, Body const &body) {
    tbb_shim::run(range, body);
}
template <class Range, class Body, class Partitioner>
void parallel_for(Range const &range, Body const &body, Partitioner const &) {
    tbb_shim::run(range, body);
}

} // namespace tbb
