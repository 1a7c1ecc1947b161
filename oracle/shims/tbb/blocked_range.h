// Minimal stand-in for oneTBB's blocked_range / split (TEST INFRASTRUCTURE).
//
// smallgwn's CPU reference code (tests/reference_cpu.cuh, tests/reference_hdk.cuh and the vendored
// SideFX HDK solid-angle tree) is written against oneTBB, which this machine does not have. This
// header and tbb/parallel_for.h provide the few names that code uses, with the same semantics:
// a half-open range [begin, end) with a grain size, and a splitting constructor that moves the
// upper half of a range into the new one.
#pragma once

#include <cstddef>

namespace tbb {

class split {};

template <class T> class blocked_range {
  public:
    using const_iterator = T;
    using size_type = std::size_t;

    blocked_range(T begin, T end, size_type grainsize = 1) : b_(begin), e_(end), g_(grainsize ? grainsize : 1) {}
    blocked_range(blocked_range &r, split) : b_(r.b_ + (r.e_ - r.b_) / 2), e_(r.e_), g_(r.g_) { r.e_ = b_; }

    T begin() const { return b_; }
    T end() const { return e_; }
    size_type size() const { return static_cast<size_type>(e_ - b_); }
    size_type grainsize() const { return g_; }
    bool empty() const { return !(b_ < e_); }
    bool is_divisible() const { return g_ < size(); }

  private:
    T b_, e_;
    size_type g_;
};

} // namespace tbb
