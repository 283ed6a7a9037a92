// Minimal stand-in for the TBB range type ProtoRay's CPU renderer uses
// (reference: sys/tasking.h:19-21, image/accum_buffer.h:109-120).
// Test infrastructure only: TBB is not installed in this image.
#pragma once

namespace tbb {

template <class T>
class blocked_range
{
    T b_, e_;

public:
    blocked_range(T b, T e) : b_(b), e_(e) {}
    T begin() const { return b_; }
    T end() const { return e_; }
    bool empty() const { return !(b_ < e_); }
};

} // namespace tbb
